// Host build of the shell element adjoint for the CPU tests: the same header
// the GPU adjoint kernel uses, compiled with g++ and exposed over flat arrays.
#include "../../openradioss_b200/csrc/shell_adjoint.cuh"
#include "../../openradioss_b200/csrc/coqini_table.h"

using namespace orb_adj;
constexpr int NP = 10;
static_assert(sizeof(ShellIn<NP>) == 103 * sizeof(double), "flat input layout");
static_assert(sizeof(ShellOut<NP>) == 89 * sizeof(double), "flat output layout");

extern "C" {
int adj_sizes(int* nin, int* nout) {
  *nin = (int)(sizeof(ShellIn<NP>) / sizeof(double));
  *nout = (int)(sizeof(ShellOut<NP>) / sizeof(double));
  return NP;
}
void adj_forward(const ShellParams* p, const double* in, double* out) {
  ShellTape<NP> t;
  ShellOut<NP> o{};
  shell_forward<NP>(*p, &ZW_TABLE[0][0], *(const ShellIn<NP>*)in, o, t);
  *(ShellOut<NP>*)out = o;
}
void adj_reverse(const ShellParams* p, const double* in, const double* outbar, double* inbar) {
  ShellTape<NP> t;
  ShellOut<NP> o{};
  ShellIn<NP> ib{};
  shell_forward<NP>(*p, &ZW_TABLE[0][0], *(const ShellIn<NP>*)in, o, t);
  shell_reverse<NP>(*p, &ZW_TABLE[0][0], *(const ShellIn<NP>*)in, t, *(const ShellOut<NP>*)outbar, ib);
  *(ShellIn<NP>*)inbar = ib;
}
}
