// ecycle_oracle.cpp -- CPU restatement of the OpenRadioss explicit element
// cycle, used ONLY as test infrastructure (the parity checker and the CPU
// baseline).  Nothing in the product links or calls this file.
//
// Parity status: the reference (Fortran, no compiler in this container) cannot
// be run here.  This restatement is pinned against the reference engine's own
// output: on the reference's QA case miniqa/RESTART/cra2 (BT shells, LAW2
// with a yield cap, 3 integration points, ISHFRAM 2, /BCS, /ADMAS, /INIVEL,
// a /VEL/TRA rigid link, two engine runs, 3375 cycles) it reproduces every
// printed digit of the listing's time, time step, time-step element,
// internal and kinetic energies (tests/test_oracle_cra2.py, fixture
// tests/golden/cra2_listing.json).  The solid path is pinned by hand-derived
// known-answer tests (tests/test_oracle_known_answers.py); no reference
// listing exercises it.
//
// Each routine follows the reference routine cited beside it, in the same
// operation order, with "my_real" = R (double for the FP64 form, float for the
// split form) and DOUBLE PRECISION where the reference declares it.  In the
// split form, geometry (Jacobian, volume, local coordinates) is evaluated in
// FP64 and cast, which matches or exceeds the reference -prec=sp build.
//
// Assembly follows Parith/ON: every element corner writes its own skyline
// slot (scumu3p.F:205-260, cupdt3.F:966-1063) and each node sums its slots in
// ascending slot order (asspar4.F:160-175).  Slots of a node are ordered by
// global element number, solids before shells (the starter's CNE order).

#include <cmath>
#include <cstring>
#include <cstdio>
#include <vector>
#include <string>
#include <algorithm>
#include <array>
#include <omp.h>
#include "../include/or_ecycle.h"

namespace {

const double EM15 = 1e-15, EM20 = 1e-20, EM30 = 1e-30;

// COQINI tables (engine/source/elements/shell/coqini.F:45-130): REAL DATA
// literals, i.e. single-precision values widened to my_real.
static const float Z01[11][11] = {
  {0.f},
  {-.5f, .5f},
  {-.5f, 0.f, .5f},
  {-.5f, -.1666667f, .1666667f, .5f},
  {-.5f, -.25f, 0.f, .25f, .5f},
  {-.5f, -.3f, -.1f, .1f, .3f, .5f},
  {-.5f, -.3333333f, -.1666667f, 0.f, .1666667f, .3333333f, .5f},
  {-.5f, -.3571429f, -.2142857f, -.0714286f, .0714286f, .2142857f, .3571429f, .5f},
  {-.5f, -.375f, -.25f, -.125f, 0.f, .125f, .25f, .375f, .5f},
  {-.5f, -.3888889f, -.2777778f, -.1666667f, -.0555555f, .0555555f, .1666667f, .2777778f, .3888889f, .5f},
  {-.5f, -.4f, -.3f, -.2f, -.1f, 0.f, .1f, .2f, .3f, .4f, .5f}};
static const float WF1[11][11] = {
  {1.f},
  {.5f, .5f},
  {.25f, .5f, .25f},
  {.1666667f, .3333333f, .3333333f, .1666667f},
  {.125f, .25f, .25f, .25f, .125f},
  {.1f, .2f, .2f, .2f, .2f, .1f},
  {.0833333f, .1666667f, .1666667f, .1666667f, .1666667f, .1666667f, .0833333f},
  {.0714286f, .1428571f, .1428571f, .1428571f, .1428571f, .1428571f, .1428571f, .0714286f},
  {.0625f, .125f, .125f, .125f, .125f, .125f, .125f, .125f, .0625f},
  {.0555556f, .1111111f, .1111111f, .1111111f, .1111111f, .1111111f, .1111111f, .1111111f, .1111111f, .0555556f},
  {.05f, .1f, .1f, .1f, .1f, .1f, .1f, .1f, .1f, .1f, .05f}};
static const float WM1[11][11] = {
  {0.f},
  {-.0833333f, .0833333f},
  {-.0833333f, 0.f, .0833333f},
  {-.0648148f, -.0555556f, .0555556f, .0648148f},
  {-.0520833f, -.0625f, 0.f, .0625f, .0520833f},
  {-.0433333f, -.06f, -.02f, .02f, .06f, .0433333f},
  {-.037037f, -.0555556f, -.0277778f, 0.f, .0277778f, .0555556f, .037037f},
  {-.0323129f, -.0510204f, -.0306122f, -.0102041f, .0102041f, .0306122f, .0510204f, .0323129f},
  {-.0286458f, -.046875f, -.03125f, -.015625f, 0.f, .015625f, .03125f, .046875f, .0286458f},
  {-.0257202f, -.0432099f, -.0308642f, -.0185185f, -.0061728f, .0061728f, .0185185f, .0308642f, .0432099f, .0257202f},
  {-.0233333f, -.04f, -.03f, -.02f, -.01f, 0.f, .01f, .02f, .03f, .04f, .0233333f}};

template <class R> inline R sgn(R a, R b) { return b >= R(0) ? std::fabs(a) : -std::fabs(a); }

struct Part;

template <class R>
struct HexGroup {
  int part, nel, gofs;        // gofs: global element number of the first element
  std::vector<int> ix;        // 8*nel, 0-based node index within the part
  or_material mat; or_solid_prop prop;
  std::vector<R> sig;         // 6*nel component-major
  std::vector<R> eint, rho, qvis, off, pla, epsd, vol0;
  std::vector<double> vol0dp;
  std::vector<long> iads;     // 8*nel skyline slot per corner
};

template <class R>
struct ShellGroup {
  int part, nel, gofs;
  std::vector<int> ix;        // 4*nel
  or_material mat; or_shell_prop prop;
  std::vector<R> thke, thk, hourg, eint, sig, pla; // hourg 3*nel, eint 2*nel, sig npt*5*nel, pla npt*nel
  std::vector<R> jca;         // optional per-element yield stress A (LAW2); empty = uniform
  std::vector<long> iadc;     // 4*nel
};

template <class R>
struct PartData {
  int numnod;
  std::vector<double> x, d;   // 3*numnod (XDP, DDP)
  std::vector<R> v, vr, a, ar, ms, in;
  std::vector<int> icodt, icodr;
  std::vector<long> adsky;    // numnod+1
  std::vector<R> fsky;        // 8*lsky
  long lsky = 0;
  int nel_solid = 0, nel_shell = 0;
  double ehour = 0, wplast = 0, wext = 0;
  std::vector<int> iskew;     // per node skew frame of the /BCS codes, -1 = global
  long lsky_elem = 0;         // slots of the elements; load slots follow
  double ekin = 0, ekinr = 0;
};

// time function (/FUNCT) and loads (/CLOAD, /PLOAD): force.F90
struct Func { std::vector<double> x, y; };
struct CLoad { int part, node, dir, skew, func; double fcx, fcy; long slot; };     // one per node
struct PLoad { int part, n[4], func; double fcx, fcy; long slot[4]; };           // one per segment

// rigid velocity link (/VEL/TRA, /VEL/ROT): frelnk.F:75-101, rlink1.F
struct RLink {
  int part, ic, icr;
  std::vector<int> nodes;     // 0-based, in the card's order
};

// rigid body (/RBODY after the starter's INIRBY): main node, secondary nodes, and
// RBY(1:12) = principal axes e1, e2, e3 (RBY(1:3), (4:6), (7:9)) and inertias
template <class R>
struct RBody {
  int part, master;
  std::vector<int> slaves;    // 0-based
  R rby[12];
};

template <class R>
struct Model {
  typedef R real_t;
  or_ecycle_config cfg;
  std::vector<PartData<R>> parts;
  std::vector<HexGroup<R>> hex;
  std::vector<ShellGroup<R>> shell;
  std::vector<RLink> rlinks;
  std::vector<RBody<R>> rbodies;
  std::vector<Func> funcs;
  std::vector<std::array<double, 9>> skews;
  std::vector<CLoad> cloads;
  std::vector<PLoad> ploads;
  bool finalized = false;
  std::string err;
  int errcode = 0, errindex = -1;
};

// ----------------------------------------------------------------------------
// Skyline construction: the starter's node->element list (CNE) gives, per node,
// the solids in ascending order then the shells in ascending order.
// ----------------------------------------------------------------------------
template <class R>
void build_skyline(Model<R>& m) {
  for (size_t p = 0; p < m.parts.size(); ++p) {
    PartData<R>& P = m.parts[p];
    std::vector<long> cnt(P.numnod + 1, 0);
    for (auto& g : m.hex) if (g.part == (int)p) for (int i = 0; i < 8 * g.nel; ++i) cnt[g.ix[i] + 1]++;
    for (auto& g : m.shell) if (g.part == (int)p) for (int i = 0; i < 4 * g.nel; ++i) cnt[g.ix[i] + 1]++;
    for (auto& c : m.cloads) if (c.part == (int)p) cnt[c.node + 1]++;
    for (auto& q : m.ploads) if (q.part == (int)p) for (int k = 0; k < (q.n[3] >= 0 ? 4 : 3); ++k) cnt[q.n[k] + 1]++;
    P.adsky.assign(P.numnod + 1, 0);
    for (int n = 0; n < P.numnod; ++n) P.adsky[n + 1] = P.adsky[n] + cnt[n + 1];
    P.lsky = P.adsky[P.numnod];
    std::vector<long> next(P.adsky.begin(), P.adsky.end() - 1);
    for (auto& g : m.hex) if (g.part == (int)p) {
      g.iads.assign(8 * g.nel, 0);
      for (int e = 0; e < g.nel; ++e) for (int k = 0; k < 8; ++k) g.iads[8 * e + k] = next[g.ix[8 * e + k]]++;
    }
    for (auto& g : m.shell) if (g.part == (int)p) {
      g.iadc.assign(4 * g.nel, 0);
      for (int e = 0; e < g.nel; ++e) for (int k = 0; k < 4; ++k) g.iadc[4 * e + k] = next[g.ix[4 * e + k]]++;
    }
    // load slots: after every element slot of their node, in load order
    for (auto& c : m.cloads) if (c.part == (int)p) c.slot = next[c.node]++;
    for (auto& q : m.ploads) if (q.part == (int)p)
      for (int k = 0; k < (q.n[3] >= 0 ? 4 : 3); ++k) q.slot[k] = next[q.n[k]]++;
    P.fsky.assign(8 * P.lsky, R(0));
    if (P.iskew.empty()) P.iskew.assign(P.numnod, -1);
  }
}

// ----------------------------------------------------------------------------
// SFORC3 chain for one 8-node 1-point hexa, JCVT=0, JLAG=1, JHBE=1, ISMSTR=4.
// ----------------------------------------------------------------------------
template <class R>
int hex_element(const Model<R>& m, HexGroup<R>& g, PartData<R>& P, int i, double dt1d,
                double& dt2t_out, double& ehou_out, double& wpla_out) {
  const bool split = (m.cfg.precision == OR_PREC_SPLIT);
  const R DT1 = R(dt1d);
  const or_material& mt = g.mat;
  int nc[8];
  for (int k = 0; k < 8; ++k) nc[k] = g.ix[8 * i + k];
  // SCOOR3 (scoor3.F:127-180, 289-312): XD in DOUBLE PRECISION, V in my_real
  double XD[8], YD[8], ZD[8];
  R VX[8], VY[8], VZ[8];
  for (int k = 0; k < 8; ++k) {
    XD[k] = P.x[3 * nc[k]]; YD[k] = P.x[3 * nc[k] + 1]; ZD[k] = P.x[3 * nc[k] + 2];
    VX[k] = P.v[3 * nc[k]]; VY[k] = P.v[3 * nc[k] + 1]; VZ[k] = P.v[3 * nc[k] + 2];
  }
  const R OFFG = g.off[i];
  const R OFF = std::fabs(OFFG);   // ISMSTR<=4, |OFFG|<=1 branch
  // SRCOOR3 (srcoor3.F, JCVT /= 0, ISORTH = 0, |OFFG| <= 1): the convected frame
  // R = [e1 e2 e3] of SREPISO3 (srepiso3.F: differences in DOUBLE PRECISION, r, s, t
  // in my_real) and SORTHO3 (sortho3.F: normalise, three symmetric corrections,
  // then e3 = e1 x v, e2 = e3 x e1); coordinates XD (DOUBLE PRECISION) and
  // velocities (my_real, SRROTA3) expressed in it
  const bool corot = g.prop.jcvt != 0;
  R R11 = 1, R12 = 0, R13 = 0, R21 = 0, R22 = 1, R23 = 0, R31 = 0, R32 = 0, R33 = 1;
  if (corot) {
    const R X17 = R(XD[6] - XD[0]), X28 = R(XD[7] - XD[1]), X35 = R(XD[4] - XD[2]), X46 = R(XD[5] - XD[3]);
    const R Y17 = R(YD[6] - YD[0]), Y28 = R(YD[7] - YD[1]), Y35 = R(YD[4] - YD[2]), Y46 = R(YD[5] - YD[3]);
    const R Z17 = R(ZD[6] - ZD[0]), Z28 = R(ZD[7] - ZD[1]), Z35 = R(ZD[4] - ZD[2]), Z46 = R(ZD[5] - ZD[3]);
    const R A17 = X17 + X46, A28 = X28 + X35, B17 = Y17 + Y46, B28 = Y28 + Y35, C17 = Z17 + Z46, C28 = Z28 + Z35;
    const R rx = X17 + X28 - X35 - X46, ry = Y17 + Y28 - Y35 - Y46, rz = Z17 + Z28 - Z35 - Z46;
    const R sx = A17 + A28, sy = B17 + B28, sz = C17 + C28;
    const R tx = A17 - A28, ty = B17 - B28, tz = C17 - C28;
    auto unit = [](R x, R y, R z, R& ux, R& uy, R& uz) {
      R aa = std::sqrt(x * x + y * y + z * z);
      if (aa != R(0)) aa = R(1) / aa;
      ux = x * aa; uy = y * aa; uz = z * aa;
    };
    R Ux, Uy, Uz, Vx, Vy, Vz, Wx, Wy, Wz;
    unit(rx, ry, rz, Ux, Uy, Uz);
    unit(sx, sy, sz, Vx, Vy, Vz);
    unit(tx, ty, tz, Wx, Wy, Wz);
    for (int it = 0; it < 3; ++it) {       // NITER = 3
      const R e1x = Vy * Wz - Vz * Wy + Ux, e1y = Vz * Wx - Vx * Wz + Uy, e1z = Vx * Wy - Vy * Wx + Uz;
      const R e2x = Wy * Uz - Wz * Uy + Vx, e2y = Wz * Ux - Wx * Uz + Vy, e2z = Wx * Uy - Wy * Ux + Vz;
      const R e3x = Uy * Vz - Uz * Vy + Wx, e3y = Uz * Vx - Ux * Vz + Wy, e3z = Ux * Vy - Uy * Vx + Wz;
      unit(e1x, e1y, e1z, Ux, Uy, Uz);
      unit(e2x, e2y, e2z, Vx, Vy, Vz);
      unit(e3x, e3y, e3z, Wx, Wy, Wz);
    }
    const R e1x = Ux, e1y = Uy, e1z = Uz;
    R e3x = e1y * Vz - e1z * Vy, e3y = e1z * Vx - e1x * Vz, e3z = e1x * Vy - e1y * Vx;
    unit(e3x, e3y, e3z, e3x, e3y, e3z);
    const R e2x = e3y * e1z - e3z * e1y, e2y = e3z * e1x - e3x * e1z, e2z = e3x * e1y - e3y * e1x;
    R11 = e1x; R21 = e1y; R31 = e1z; R12 = e2x; R22 = e2y; R32 = e2z; R13 = e3x; R23 = e3y; R33 = e3z;
    for (int k = 0; k < 8; ++k) {
      const double xl = double(R11) * XD[k] + double(R21) * YD[k] + double(R31) * ZD[k];
      const double yl = double(R12) * XD[k] + double(R22) * YD[k] + double(R32) * ZD[k];
      const double zl = double(R13) * XD[k] + double(R23) * YD[k] + double(R33) * ZD[k];
      XD[k] = xl; YD[k] = yl; ZD[k] = zl;
      const R vx = R11 * VX[k] + R21 * VY[k] + R31 * VZ[k];
      const R vy = R12 * VX[k] + R22 * VY[k] + R32 * VZ[k];
      const R vz = R13 * VX[k] + R23 * VY[k] + R33 * VZ[k];
      VX[k] = vx; VY[k] = vy; VZ[k] = vz;
    }
  }

  // SDERI3 (sderi3.F:103-149 Jacobian; 264-298 inverse; 302-333 hourglass projections)
  // Geometry: FP64 form = reference dp; split form evaluates it in FP64 and casts.
  typedef double G;
  G X17 = XD[6] - XD[0], X28 = XD[7] - XD[1], X35 = XD[4] - XD[2], X46 = XD[5] - XD[3];
  G Y17 = YD[6] - YD[0], Y28 = YD[7] - YD[1], Y35 = YD[4] - YD[2], Y46 = YD[5] - YD[3];
  G Z17 = ZD[6] - ZD[0], Z28 = ZD[7] - ZD[1], Z35 = ZD[4] - ZD[2], Z46 = ZD[5] - ZD[3];
  G JAC1 = X17 + X28 - X35 - X46, JAC2 = Y17 + Y28 - Y35 - Y46, JAC3 = Z17 + Z28 - Z35 - Z46;
  G X_17_46 = X17 + X46, X_28_35 = X28 + X35, Y_17_46 = Y17 + Y46, Y_28_35 = Y28 + Y35;
  G Z_17_46 = Z17 + Z46, Z_28_35 = Z28 + Z35;
  G JAC4 = X_17_46 + X_28_35, JAC5 = Y_17_46 + Y_28_35, JAC6 = Z_17_46 + Z_28_35;
  G JAC7 = X_17_46 - X_28_35, JAC8 = Y_17_46 - Y_28_35, JAC9 = Z_17_46 - Z_28_35;
  G JAC_59_68 = JAC5 * JAC9 - JAC6 * JAC8;
  G JAC_67_49 = JAC6 * JAC7 - JAC4 * JAC9;
  G JAC_48_57 = JAC4 * JAC8 - JAC5 * JAC7;
  G VOLDP = (1.0 / 64.0) * (JAC1 * JAC_59_68 + JAC2 * JAC_67_49 + JAC3 * JAC_48_57);
  G DET = VOLDP;
  if (!(OFF == R(0))) {
    if (!(DET > 0.0)) return OR_E_NEGVOL;   // SCHKJABT3 (schkjabt3.F): INEG_V=0 -> stop
  } else {
    DET = 1.0;
  }
  G DETT = (1.0 / 64.0) / DET;
  G JACI1 = DETT * JAC_59_68, JACI4 = DETT * JAC_67_49, JACI7 = DETT * JAC_48_57;
  G JACI2 = DETT * (JAC3 * JAC8 - JAC2 * JAC9);
  G JACI5 = DETT * (JAC1 * JAC9 - JAC3 * JAC7);
  G JACI8 = DETT * (JAC2 * JAC7 - JAC1 * JAC8);
  G JACI3 = DETT * (JAC2 * JAC6 - JAC3 * JAC5);
  G JACI6 = DETT * (JAC3 * JAC4 - JAC1 * JAC6);
  G JACI9 = DETT * (JAC1 * JAC5 - JAC2 * JAC4);
  G JAC12 = JACI1 + JACI2, JAC45 = JACI4 + JACI5, JAC78 = JACI7 + JACI8;
  G px1 = -JAC12 - JACI3, py1 = -JAC45 - JACI6, pz1 = -JAC78 - JACI9;
  G px2 = -JAC12 + JACI3, py2 = -JAC45 + JACI6, pz2 = -JAC78 + JACI9;
  JAC12 = JACI1 - JACI2; JAC45 = JACI4 - JACI5; JAC78 = JACI7 - JACI8;
  G px3 = JAC12 + JACI3, py3 = JAC45 + JACI6, pz3 = JAC78 + JACI9;
  G px4 = JAC12 - JACI3, py4 = JAC45 - JACI6, pz4 = JAC78 - JACI9;
  R PX[4] = {R(px1), R(px2), R(px3), R(px4)};
  R PY[4] = {R(py1), R(py2), R(py3), R(py4)};
  R PZ[4] = {R(pz1), R(pz2), R(pz3), R(pz4)};
  // hourglass mode projections (JHBE/=0)
  static const int HM[3][8] = {{1, -1, 1, -1, 1, -1, 1, -1}, {1, 1, -1, -1, -1, -1, 1, 1}, {1, -1, -1, 1, -1, 1, 1, -1}};
  R PXH[4][3];
  for (int j = 0; j < 3; ++j) {
    G HX = 0, HY = 0, HZ = 0;
    for (int k = 0; k < 8; ++k) { HX += HM[j][k] * XD[k]; HY += HM[j][k] * YD[k]; HZ += HM[j][k] * ZD[k]; }
    // reference: HX is my_real, products in my_real
    R hx = R(HX), hy = R(HY), hz = R(HZ);
    for (int a = 0; a < 4; ++a) PXH[a][j] = PX[a] * hx + PY[a] * hy + PZ[a] * hz;
  }
  const double VOLN_D = DET;
  const R VOLN = R(DET);

  // SDLEN3 + SLEN (sdlen3.F:110-166, slen.F): faces (1234)(5678)(1265)(2376)(3487)(4158)
  static const int FC[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
  R AREAM = R(EM20);
  for (int f = 0; f < 6; ++f) {
    const int* q = FC[f];
    // X13 = X3-X1 etc. in my_real (X = XD cast)
    R X13 = R(R(XD[q[2]]) - R(XD[q[0]])), X24 = R(R(XD[q[3]]) - R(XD[q[1]]));
    R Y13 = R(R(YD[q[2]]) - R(YD[q[0]])), Y24 = R(R(YD[q[3]]) - R(YD[q[1]]));
    R Z13 = R(R(ZD[q[2]]) - R(ZD[q[0]])), Z24 = R(R(ZD[q[3]]) - R(ZD[q[1]]));
    if (split) {   // split form: differences of the FP64 coordinates
      X13 = R(XD[q[2]] - XD[q[0]]); X24 = R(XD[q[3]] - XD[q[1]]);
      Y13 = R(YD[q[2]] - YD[q[0]]); Y24 = R(YD[q[3]] - YD[q[1]]);
      Z13 = R(ZD[q[2]] - ZD[q[0]]); Z24 = R(ZD[q[3]] - ZD[q[1]]);
    }
    R FS1 = X13 - X24, FT1 = X13 + X24, FS2 = Y13 - Y24, FT2 = Y13 + Y24, FS3 = Z13 - Z24, FT3 = Z13 + Z24;
    R E = FS1 * FS1 + FS2 * FS2 + FS3 * FS3;
    R F = FS1 * FT1 + FS2 * FT2 + FS3 * FT3;
    R Gm = FT1 * FT1 + FT2 * FT2 + FT3 * FT3;
    R AREA = E * Gm - F * F;
    AREAM = std::max(AREA, AREAM);
  }
  const R DELTAX = R(4) * VOLN / std::sqrt(AREAM);

  // SDEFO3 (sdefo3.F:114-170), JHBE=1 branch
  R VX17 = VX[0] - VX[6], VX28 = VX[1] - VX[7], VX35 = VX[2] - VX[4], VX46 = VX[3] - VX[5];
  R VY17 = VY[0] - VY[6], VY28 = VY[1] - VY[7], VY35 = VY[2] - VY[4], VY46 = VY[3] - VY[5];
  R VZ17 = VZ[0] - VZ[6], VZ28 = VZ[1] - VZ[7], VZ35 = VZ[2] - VZ[4], VZ46 = VZ[3] - VZ[5];
  R DXX = PX[0] * VX17 + PX[1] * VX28 + PX[2] * VX35 + PX[3] * VX46;
  R DYY = PY[0] * VY17 + PY[1] * VY28 + PY[2] * VY35 + PY[3] * VY46;
  R DZZ = PZ[0] * VZ17 + PZ[1] * VZ28 + PZ[2] * VZ35 + PZ[3] * VZ46;
  R DXY = PY[0] * VX17 + PY[1] * VX28 + PY[2] * VX35 + PY[3] * VX46;
  R DXZ = PZ[0] * VX17 + PZ[1] * VX28 + PZ[2] * VX35 + PZ[3] * VX46;
  R DYX = PX[0] * VY17 + PX[1] * VY28 + PX[2] * VY35 + PX[3] * VY46;
  R DYZ = PZ[0] * VY17 + PZ[1] * VY28 + PZ[2] * VY35 + PZ[3] * VY46;
  R DZX = PX[0] * VZ17 + PX[1] * VZ28 + PX[2] * VZ35 + PX[3] * VZ46;
  R DZY = PY[0] * VZ17 + PY[1] * VZ28 + PY[2] * VZ35 + PY[3] * VZ46;
  const R DT1D2 = R(0.5) * DT1;
  R D4 = DXY + DYX, D5 = DYZ + DZY, D6 = DXZ + DZX;
  R WZZ = DT1D2 * (DYX - DXY), WYY = DT1D2 * (DXZ - DZX), WXX = DT1D2 * (DZY - DYZ);

  // SRHO3 (srho3.F:122-156 Lagrangian; IRESP branch :230-245 for the split form)
  const R RHO0 = R(mt.rho0);
  R RHON = g.rho[i];
  const R RHON_OLD = RHON;
  const R VOLO = g.vol0[i];
  R DIVDE = DT1 * (DXX + DYY + DZZ); (void)DIVDE;
  R DVOL = VOLN - (RHO0 / RHON) * VOLO;
  RHON = RHO0 * (VOLO / VOLN);
  R EINT = g.eint[i] * VOLO;
  R AMU;
  if (split) {
    const double V0 = g.vol0dp[i];
    DVOL = R(VOLN_D - (double(RHO0) / double(RHON_OLD)) * V0);
    RHON = R(double(RHO0) * (V0 / VOLN_D));
    AMU = R(V0 / VOLN_D - 1.0);
  } else {
    AMU = RHON / RHO0 - R(1);          // mmain.F90: amu = rho/rho0 - 1 (laws 1, 2)
  }

  // SROTA3 (srota3.F:81-91)
  R S1 = g.sig[0 * g.nel + i], S2 = g.sig[1 * g.nel + i], S3 = g.sig[2 * g.nel + i];
  R S4 = g.sig[3 * g.nel + i], S5 = g.sig[4 * g.nel + i], S6 = g.sig[5 * g.nel + i];
  R SIG[6];
  if (corot) {          // SRMALLA3 (srmall3.F): the convected-frame stress, not rotated
    SIG[0] = S1; SIG[1] = S2; SIG[2] = S3; SIG[3] = S4; SIG[4] = S5; SIG[5] = S6;
  } else {
    R Q1 = R(2) * S4 * WZZ, Q2 = R(2) * S6 * WYY, Q3 = R(2) * S5 * WXX;
    SIG[0] = S1 - Q1 + Q2;
    SIG[1] = S2 + Q1 - Q3;
    SIG[2] = S3 - Q2 + Q3;
    SIG[3] = S4 + WZZ * (S1 - S2) + WYY * S5 - WXX * S6;
    SIG[4] = S5 + WXX * (S2 - S3) + WZZ * S6 - WYY * S4;
    SIG[5] = S6 + WYY * (S3 - S1) + WXX * S4 - WZZ * S5;
  }
  // MMAIN preamble (mmain.F90:690-725)
  const R VOL_AVG = VOLN - R(0.5) * DVOL;
  const R RHOREF = RHON; (void)RHOREF;
  const R QOLD = g.qvis[i];
  const R D1 = DXX, D2 = DYY, D3 = DZZ;
  R SSP, PNEW, QNEW, DTX, STI;
  R DPLA = 0, SIGY = 0;
  R G0 = (mt.law == OR_LAW_ELASTIC) ? R(mt.shear) : R(mt.shear);
  R Gm = G0 * OFF;
  R G1 = DT1 * Gm, G2 = R(2) * G1;
  R AJ2 = 0;
  {
    // deviatoric predictor, common to m1law.F:124-140 and m2law.F:187-200
    R KB = (mt.law == OR_LAW_ELASTIC) ? R(mt.bulk) : R(mt.bulk);
    SSP = std::sqrt((R(1.333) * Gm + KB) / RHO0);
    R P = -(SIG[0] + SIG[1] + SIG[2]) / R(3);
    R DAV = -(D1 + D2 + D3) / R(3);
    if (mt.law == OR_LAW_ELASTIC) {
      P = -R(1.0 / 3.0) * (SIG[0] + SIG[1] + SIG[2]);
      DAV = -R(1.0 / 3.0) * (D1 + D2 + D3);
    } else {
      P = -R(1.0 / 3.0) * (SIG[0] + SIG[1] + SIG[2]);
      DAV = -R(1.0 / 3.0) * (D1 + D2 + D3);
    }
    SIG[0] = SIG[0] + P + G2 * (D1 + DAV);
    SIG[1] = SIG[1] + P + G2 * (D2 + DAV);
    SIG[2] = SIG[2] + P + G2 * (D3 + DAV);
    SIG[3] = SIG[3] + G1 * D4;
    SIG[4] = SIG[4] + G1 * D5;
    SIG[5] = SIG[5] + G1 * D6;
  }
  if (mt.law == OR_LAW_JOHNSON_COOK) {
    // m2law.F:197-352 (CC=0, FISOKIN=0, IFORM=0, TSTAR=0 -> EPD=1)
    AJ2 = R(0.5) * (SIG[0] * SIG[0] + SIG[1] * SIG[1] + SIG[2] * SIG[2]) + SIG[3] * SIG[3] + SIG[4] * SIG[4] + SIG[5] * SIG[5];
    AJ2 = std::sqrt(R(3) * AJ2);
    // MSTRAIN_RATE (mstrain_rate.F), ISRATE=0, IDEV=0
    {
      R E1 = D1, E2 = D2, E3 = D3, E4 = R(0.5) * D4, E5 = R(0.5) * D5, E6 = R(0.5) * D6;
      R EPSP = E1 * E1 + E2 * E2 + E3 * E3 + R(2) * (E4 * E4 + E5 * E5 + E6 * E6);
      g.epsd[i] = std::sqrt(EPSP);
    }
    const R CA = R(mt.jc_a), CB = R(mt.jc_b), CN = R(mt.jc_n), EPMX = R(mt.epsmax), SIGMX = R(mt.sigmax);
    R EPXE = g.pla[i];
    const R EPD = R(1);
    R AK, QH;
    if (CN == R(1)) {
      AK = CA + CB * EPXE;
      QH = CB * EPD;
    } else if (EPXE > R(0)) {
      AK = CA + CB * std::pow(EPXE, CN);
      if (CN > R(1)) QH = (CB * CN * std::pow(EPXE, CN - R(1))) * EPD;
      else QH = (CB * CN / std::pow(EPXE, R(1) - CN)) * EPD;
    } else {
      AK = CA; QH = 0;
    }
    AK = AK * EPD;
    if (SIGMX < AK) { AK = SIGMX; QH = 0; }
    SIGY = AK;
    if (EPXE > EPMX) { AK = 0; QH = 0; }
    R SCALE = std::min(R(1), AK / std::max(AJ2, R(EM15)));
    DPLA = (R(1) - SCALE) * AJ2 / std::max(R(3) * Gm + QH, R(EM15));
    AK = AK + DPLA * QH;
    SCALE = std::min(R(1), AK / std::max(AJ2, R(EM15)));
    for (int c = 0; c < 6; ++c) SIG[c] = SCALE * SIG[c];
    EPXE = EPXE + DPLA;
    g.pla[i] = EPXE;
    SIGY = std::max(SIGY, AK);
  }
  // MQVISCB (mqviscb.F:139-354), FACQ=1, VISI=1, NPG=1, CNS1=CNS2=0, VIS=0, VD2=0
  {
    R DD = -D1 - D2 - D3;
    R CX = SSP;
    R AL = 0, AD = 0;
    if (OFF == R(1)) {
      AL = (VOLN > R(0)) ? R(std::pow(VOLN, R(1) / R(3))) : R(0);
      AD = std::max(R(0), DD);
    }
    const R QA = R(g.prop.qa), QB = R(g.prop.qb);
    R QAA = QA * QA * AD;
    R QX = QB * SSP + AL * QAA;
    QNEW = RHON * AD * AL * (QAA * AL + QB * SSP);
    R SSP_EQ = std::max(R(EM20), QX + std::sqrt(QX * QX + CX * CX));
    DTX = DELTAX / SSP_EQ;
    R TIDT = R(1) / DTX;
    STI = (RHON * TIDT) * (VOLN * TIDT);
    if (OFF == R(0) || OFFG < R(0)) STI = 0;
    DTX = R(m.cfg.dtfac_solid) * DTX;
    if (VOLN > R(0) && OFF != R(0) && OFFG >= R(0)) {
      if (double(DTX) <= m.cfg.dtmin_solid) return OR_E_DTMIN;
      dt2t_out = std::min(dt2t_out, double(DTX));
    }
  }
  // pressure and energy (m1law.F:172-190, m2law.F:434-461)
  const R DTA = R(0.5) * DT1;
  if (mt.law == OR_LAW_ELASTIC) {
    PNEW = R(mt.bulk) * AMU;
    SIG[0] = (SIG[0] - PNEW) * OFF; SIG[1] = (SIG[1] - PNEW) * OFF; SIG[2] = (SIG[2] - PNEW) * OFF;
    SIG[3] = SIG[3] * OFF; SIG[4] = SIG[4] * OFF; SIG[5] = SIG[5] * OFF;
    R P2 = -(S1 + SIG[0] + S2 + SIG[1] + S3 + SIG[2]) * R(1.0 / 3.0);
    R E1 = D1 * (S1 + SIG[0] + P2), E2 = D2 * (S2 + SIG[1] + P2), E3 = D3 * (S3 + SIG[2] + P2);
    R E4 = D4 * (S4 + SIG[3]), E5 = D5 * (S5 + SIG[4]), E6 = D6 * (S6 + SIG[5]);
    R EINC = VOL_AVG * (E1 + E2 + E3 + E4 + E5 + E6) * DTA - R(0.5) * DVOL * (QOLD + QNEW + P2);
    EINT = (EINT + EINC * OFF) / std::max(R(EM15), VOLO);
  } else {
    PNEW = R(mt.bulk) * AMU;
    SIG[0] = (SIG[0] - PNEW) * OFF; SIG[1] = (SIG[1] - PNEW) * OFF; SIG[2] = (SIG[2] - PNEW) * OFF;
    SIG[3] = SIG[3] * OFF; SIG[4] = SIG[4] * OFF; SIG[5] = SIG[5] * OFF;
    R E1 = D1 * (S1 + SIG[0]), E2 = D2 * (S2 + SIG[1]), E3 = D3 * (S3 + SIG[2]);
    R E4 = D4 * (S4 + SIG[3]), E5 = D5 * (S5 + SIG[4]), E6 = D6 * (S6 + SIG[5]);
    R EINC = VOL_AVG * (E1 + E2 + E3 + E4 + E5 + E6) * DTA - R(0.5) * DVOL * (QOLD + QNEW);
    EINT = (EINT + EINC * OFF) / std::max(R(EM15), VOLO);
    wpla_out += double(SIGY) * double(DPLA) * double(VOLN);
  }
  for (int c = 0; c < 6; ++c) g.sig[c * g.nel + i] = SIG[c];
  g.eint[i] = EINT;
  g.rho[i] = RHON;
  g.qvis[i] = QNEW;

  // SHVIS3 (shvis3.F:156-424), INVSTR>=35, non fluid, ISMSTR=4, JHBE>=1
  R F[3][8];
  {
    R CAQ = R(0.25) * OFF * R(g.prop.qh);
    R FCL = CAQ * RHON * std::pow(VOLN, R(2) / R(3));
    R FCQ = FCL * CAQ * R(100);
    FCL = FCL * SSP;
    R Gv[3][8];
    for (int j = 0; j < 3; ++j) {
      // G1j = 1-PX1Hj, G2j = +-1-PX2Hj, ... (sign pattern of mode j)
      const int* s = HM[j];
      Gv[j][0] = R(s[0]) - PXH[0][j];
      Gv[j][1] = R(s[1]) - PXH[1][j];
      Gv[j][2] = R(s[2]) - PXH[2][j];
      Gv[j][3] = R(s[3]) - PXH[3][j];
      Gv[j][4] = R(s[4]) + PXH[2][j];
      Gv[j][5] = R(s[5]) + PXH[3][j];
      Gv[j][6] = R(s[6]) + PXH[0][j];
      Gv[j][7] = R(s[7]) + PXH[1][j];
    }
    static const int H4[8] = {1, -1, 1, -1, -1, 1, -1, 1};
    R HGX[4], HGY[4], HGZ[4];
    for (int j = 0; j < 3; ++j) {
      R hx = 0, hy = 0, hz = 0;
      hx = Gv[j][0] * VX[0] + Gv[j][1] * VX[1] + Gv[j][2] * VX[2] + Gv[j][3] * VX[3] + Gv[j][4] * VX[4] + Gv[j][5] * VX[5] + Gv[j][6] * VX[6] + Gv[j][7] * VX[7];
      hy = Gv[j][0] * VY[0] + Gv[j][1] * VY[1] + Gv[j][2] * VY[2] + Gv[j][3] * VY[3] + Gv[j][4] * VY[4] + Gv[j][5] * VY[5] + Gv[j][6] * VY[6] + Gv[j][7] * VY[7];
      hz = Gv[j][0] * VZ[0] + Gv[j][1] * VZ[1] + Gv[j][2] * VZ[2] + Gv[j][3] * VZ[3] + Gv[j][4] * VZ[4] + Gv[j][5] * VZ[5] + Gv[j][6] * VZ[6] + Gv[j][7] * VZ[7];
      HGX[j] = hx; HGY[j] = hy; HGZ[j] = hz;
    }
    HGX[3] = VX[0] - VX[1] + VX[2] - VX[3] - VX[4] + VX[5] - VX[6] + VX[7];
    HGY[3] = VY[0] - VY[1] + VY[2] - VY[3] - VY[4] + VY[5] - VY[6] + VY[7];
    HGZ[3] = VZ[0] - VZ[1] + VZ[2] - VZ[3] - VZ[4] + VZ[5] - VZ[6] + VZ[7];
    R HX[4], HY[4], HZ[4];
    for (int j = 0; j < 4; ++j) {
      HX[j] = HGX[j] * (FCL + std::fabs(HGX[j]) * FCQ);
      HY[j] = HGY[j] * (FCL + std::fabs(HGY[j]) * FCQ);
      HZ[j] = HGZ[j] * (FCL + std::fabs(HGZ[j]) * FCQ);
    }
    for (int k = 0; k < 8; ++k) {
      F[0][k] = -Gv[0][k] * HX[0] - Gv[1][k] * HX[1] - Gv[2][k] * HX[2] - R(H4[k]) * HX[3];
      F[1][k] = -Gv[0][k] * HY[0] - Gv[1][k] * HY[1] - Gv[2][k] * HY[2] - R(H4[k]) * HY[3];
      F[2][k] = -Gv[0][k] * HZ[0] - Gv[1][k] * HZ[1] - Gv[2][k] * HZ[2] - R(H4[k]) * HZ[3];
    }
    R EHOU = DT1 * (HZ[0] * HGZ[0] + HZ[1] * HGZ[1] + HZ[2] * HGZ[2] + HZ[3] * HGZ[3] +
                    HX[0] * HGX[0] + HX[1] * HGX[1] + HX[2] * HGX[2] + HX[3] * HGX[3] +
                    HY[0] * HGY[0] + HY[1] * HGY[1] + HY[2] * HGY[2] + HY[3] * HGY[3]);
    ehou_out += double(EHOU);
  }
  // SFINT3 (sfint3.F:256-321)
  {
    R sS1 = (SIG[0] - QNEW) * VOLN, sS2 = (SIG[1] - QNEW) * VOLN, sS3 = (SIG[2] - QNEW) * VOLN;
    R sS4 = SIG[3] * VOLN, sS5 = SIG[4] * VOLN, sS6 = SIG[5] * VOLN;
    static const int PAIR[4][2] = {{0, 6}, {1, 7}, {2, 4}, {3, 5}};
    for (int a = 0; a < 4; ++a) {
      int n1 = PAIR[a][0], n2 = PAIR[a][1];
      R FINT = sS1 * PX[a] + sS4 * PY[a] + sS6 * PZ[a];
      F[0][n1] -= FINT; F[0][n2] += FINT;
      FINT = sS2 * PY[a] + sS4 * PX[a] + sS5 * PZ[a];
      F[1][n1] -= FINT; F[1][n2] += FINT;
      FINT = sS3 * PZ[a] + sS6 * PX[a] + sS5 * PY[a];
      F[2][n1] -= FINT; F[2][n2] += FINT;
    }
  }
  // SRROTA3 with R transposed (sforc3.F:1603-1614): forces back to the global frame
  if (corot) {
    for (int k = 0; k < 8; ++k) {
      const R fx = R11 * F[0][k] + R12 * F[1][k] + R13 * F[2][k];
      const R fy = R21 * F[0][k] + R22 * F[1][k] + R23 * F[2][k];
      const R fz = R31 * F[0][k] + R32 * F[1][k] + R33 * F[2][k];
      F[0][k] = fx; F[1][k] = fy; F[2][k] = fz;
    }
  }
  // SCUMU3P (scumu3p.F:195-260)
  STI = R(0.25) * STI;
  for (int k = 0; k < 8; ++k) {
    long s = g.iads[8 * i + k];
    R* f = &P.fsky[8 * s];
    f[0] = F[0][k]; f[1] = F[1][k]; f[2] = F[2][k];
    f[3] = 0; f[4] = 0; f[5] = 0; f[6] = STI; f[7] = 0;
  }
  return OR_OK;
}

// Engine IHBE (IPARG(23)) of a group from the starter's Ishell: hm_read_prop01.F:
// 176 (0 -> the default, 1 here), 246-250 (one point: Ishell 0 and 2 -> 1),
// 305-315 (GEO(171): 1 -> 1, 2 -> 0, 3 -> 2, 4 -> 4), cgrtails.F:553, 949.
inline int shell_ihbe(int ishell, int npt) {
  if (ishell == 0) ishell = 1;
  if (npt == 1 && ishell == 2) ishell = 1;
  return ishell == 1 ? 1 : ishell == 2 ? 0 : ishell == 3 ? 2 : 4;
}

// ----------------------------------------------------------------------------
// CFORC3 chain for one 4-node BT shell, Ishell 1..4 (IHBE 1, 0, 2, 4), ISMSTR=2,
// ISHFRAM=0 or 2.
// ----------------------------------------------------------------------------
template <class R>
int shell_element(const Model<R>& m, ShellGroup<R>& g, PartData<R>& P, int i, double dt1d,
                  double& dt2t_out, double& ehou_out, double& wpla_out) {
  const bool split = (m.cfg.precision == OR_PREC_SPLIT);
  const R DT1 = R(dt1d);
  const or_material& mt = g.mat;
  const or_shell_prop& pr = g.prop;
  const int npt = pr.npt, nel = g.nel;
  const int IHBE = shell_ihbe(pr.ishell, npt);
  int nc[4];
  for (int k = 0; k < 4; ++k) nc[k] = g.ix[4 * i + k];
  // CCOOR3 (ccoor3.F): X (my_real), V, VR
  double XG[4], YG[4], ZG[4];
  R VL[4][3], VRL[4][3];
  for (int k = 0; k < 4; ++k) {
    XG[k] = P.x[3 * nc[k]]; YG[k] = P.x[3 * nc[k] + 1]; ZG[k] = P.x[3 * nc[k] + 2];
    if (!split) { XG[k] = double(R(XG[k])); YG[k] = double(R(YG[k])); ZG[k] = double(R(ZG[k])); }
    for (int c = 0; c < 3; ++c) { VL[k][c] = P.v[3 * nc[k] + c]; VRL[k][c] = P.vr[3 * nc[k] + c]; }
  }
  const R OFF = std::min(R(1), R(1));   // OFFG = 1 (no deletion on the path)
  // coordinate differences: my_real in the reference; FP64 then cast in the split form
  auto dif = [&](const double* a, int p, int q) -> R { return split ? R(a[p] - a[q]) : R(R(a[p]) - R(a[q])); };
  // CNVEC3 (cnvec3.F:66-140), ISHFRAM=0 or 2
  R E1X, E1Y, E1Z, E2X, E2Y, E2Z, E3X, E3Y, E3Z;
  {
    R X21 = dif(XG, 1, 0), X32 = dif(XG, 2, 1), X34 = dif(XG, 2, 3), X41 = dif(XG, 3, 0);
    R Y21 = dif(YG, 1, 0), Y32 = dif(YG, 2, 1), Y34 = dif(YG, 2, 3), Y41 = dif(YG, 3, 0);
    R Z21 = dif(ZG, 1, 0), Z32 = dif(ZG, 2, 1), Z34 = dif(ZG, 2, 3), Z41 = dif(ZG, 3, 0);
    E1X = X21 + X34; E1Y = Y21 + Y34; E1Z = Z21 + Z34;
    E2X = X32 + X41; E2Y = Y32 + Y41; E2Z = Z32 + Z41;
    E3X = E1Y * E2Z - E1Z * E2Y; E3Y = E1Z * E2X - E1X * E2Z; E3Z = E1X * E2Y - E1Y * E2X;
    if (pr.ishfram == 2) {
      // cnvec3.F:82-106: E1 = |E2|^2 E1 + E2 x E3 (E3 not yet normalised)
      R SUMA = E2X * E2X + E2Y * E2Y + E2Z * E2Z;
      E1X = E1X * SUMA + E2Y * E3Z - E2Z * E3Y;
      E1Y = E1Y * SUMA + E2Z * E3X - E2X * E3Z;
      E1Z = E1Z * SUMA + E2X * E3Y - E2Y * E3X;
      SUMA = E1X * E1X + E1Y * E1Y + E1Z * E1Z;
      SUMA = R(1) / std::max(std::sqrt(SUMA), R(EM20));
      E1X *= SUMA; E1Y *= SUMA; E1Z *= SUMA;
      SUMA = E3X * E3X + E3Y * E3Y + E3Z * E3Z;
      SUMA = R(1) / std::max(std::sqrt(SUMA), R(EM20));
      E3X *= SUMA; E3Y *= SUMA; E3Z *= SUMA;
      E2X = E3Y * E1Z - E3Z * E1Y; E2Y = E3Z * E1X - E3X * E1Z; E2Z = E3X * E1Y - E3Y * E1X;
      SUMA = E2X * E2X + E2Y * E2Y + E2Z * E2Z;
      SUMA = R(1) / std::max(std::sqrt(SUMA), R(EM20));
      E2X *= SUMA; E2Y *= SUMA; E2Z *= SUMA;
    } else {
    R SUMA = E3X * E3X + E3Y * E3Y + E3Z * E3Z;
    SUMA = R(1) / std::max(std::sqrt(SUMA), R(EM20));
    E3X *= SUMA; E3Y *= SUMA; E3Z *= SUMA;
    R S1 = E1X * E1X + E1Y * E1Y + E1Z * E1Z;
    R S2 = E2X * E2X + E2Y * E2Y + E2Z * E2Z;
    SUMA = std::sqrt(S1 / S2);
    E1X = E1X + (E2Y * E3Z - E2Z * E3Y) * SUMA;
    E1Y = E1Y + (E2Z * E3X - E2X * E3Z) * SUMA;
    E1Z = E1Z + (E2X * E3Y - E2Y * E3X) * SUMA;
    SUMA = E1X * E1X + E1Y * E1Y + E1Z * E1Z;
    SUMA = R(1) / std::max(std::sqrt(SUMA), R(EM20));
    E1X *= SUMA; E1Y *= SUMA; E1Z *= SUMA;
    E2X = E3Y * E1Z - E3Z * E1Y; E2Y = E3Z * E1X - E3X * E1Z; E2Z = E3X * E1Y - E3Y * E1X;
    }
  }
  // CDERI3 (cderi3.F:87-190)
  R X2, X3, X4, Y2, Y3, Y4, Z2;
  {
    R X21GA = dif(XG, 1, 0), Y21GA = dif(YG, 1, 0), Z21GA = dif(ZG, 1, 0);
    R X31GA = dif(XG, 2, 0), Y31GA = dif(YG, 2, 0), Z31GA = dif(ZG, 2, 0);
    R X41GA = dif(XG, 3, 0), Y41GA = dif(YG, 3, 0), Z41GA = dif(ZG, 3, 0);
    X2 = E1X * X21GA + E1Y * Y21GA + E1Z * Z21GA;
    Y2 = E2X * X21GA + E2Y * Y21GA + E2Z * Z21GA;
    Y3 = E2X * X31GA + E2Y * Y31GA + E2Z * Z31GA;
    X3 = E1X * X31GA + E1Y * Y31GA + E1Z * Z31GA;
    X4 = E1X * X41GA + E1Y * Y41GA + E1Z * Z41GA;
    Y4 = E2X * X41GA + E2Y * Y41GA + E2Z * Z41GA;
    Z2 = E3X * X21GA + E3Y * Y21GA + E3Z * Z21GA;
  }
  R PX1 = R(0.5) * (Y2 - Y4), PY1 = R(0.5) * (X4 - X2), PX2 = R(0.5) * Y3, PY2 = -R(0.5) * X3;
  R AREA = std::max(R(2) * (PY2 * PX1 - PY1 * PX2), R(EM20));
  R VHX = (-X2 + X3 - X4) / AREA, VHY = (-Y2 + Y3 - Y4) / AREA;
  // CCOEF3 (ccoef3.F:66-160)
  R THK0 = g.thke[i];
  const R VOL00 = THK0 * AREA; (void)VOL00;
  if (pr.ithk > 0) THK0 = g.thk[i];
  const R VOL0 = THK0 * AREA;
  const R THK02 = THK0 * THK0;
  const R RHO = R(mt.rho0), YM = R(mt.young), NU = R(mt.nu), GG = R(mt.shear);
  const R A11 = R(mt.a11), A12 = R(mt.a12), SSP = R(mt.ssp_shell);
  const R H1 = R(pr.hm), H2 = R(pr.hf), H3 = R(pr.hr);
  const R SHF = (npt == 1) ? R(0) : R(pr.shf);
  const R GS = GG * SHF;
  // CDLEN3 (cdlen3.F:69-121), IHBE/=0, INVSTR>=35
  R ALDT;
  {
    R AL1 = X2 * X2 + Y2 * Y2;
    R AL2 = (X3 - X2) * (X3 - X2) + (Y3 - Y2) * (Y3 - Y2);
    R AL6 = X3 * X3 + Y3 * Y3;
    R AL3 = (X4 - X3) * (X4 - X3) + (Y4 - Y3) * (Y4 - Y3);
    R AL4 = X4 * X4 + Y4 * Y4;
    R AL5 = (X4 - X2) * (X4 - X2) + (Y4 - Y2) * (Y4 - Y2);
    R ALMIN = std::min(std::min(AL1, AL2), AL4);
    R ALQUAD = std::min(std::min(AL3, AL5), AL6);
    if (AL3 != R(0)) ALMIN = std::min(ALMIN, ALQUAD);
    R DTDYN = AREA * AREA / std::max(std::max(AL5, AL6), R(EM20));
    ALDT = std::max(DTDYN, ALMIN);
    R DTHOUR = R(0.5) * (ALMIN + ALDT) / std::max(H1, H2);
    if (DTHOUR < ALDT) ALDT = DTHOUR;
    ALDT = std::sqrt(ALDT);
  }
  // CDEFO3 (cdefo3.F:84-220): local velocities, then per IHBE the membrane strain
  // rates and, for IHBE 2 and 4, the warping-corrected velocities that the
  // hourglass routines use
  R VXl[4], VYl[4], VZl[4];
  for (int k = 0; k < 4; ++k) {
    VXl[k] = E1X * VL[k][0] + E1Y * VL[k][1] + E1Z * VL[k][2];
    VYl[k] = E2X * VL[k][0] + E2Y * VL[k][1] + E2Z * VL[k][2];
    VZl[k] = E3X * VL[k][0] + E3Y * VL[k][1] + E3Z * VL[k][2];
  }
  R EXX, EYY, EXY, EXZ, EYZ;
  {
    R VZ13 = VZl[0] - VZl[2], VZ24 = VZl[1] - VZl[3];
    EYZ = PY1 * VZ13 + PY2 * VZ24;
    EXZ = PX1 * VZ13 + PX2 * VZ24;
    R VX13, VX24, VY13, VY24;
    if (IHBE <= 1) {
      // cdefo3.F:103-131 (Z2 = 0 for the hourglass forces)
      Z2 = R(0);
      R DT1V4 = R(0.25) * DT1;
      R TMP2A = PY2 + PY1;
      R TMP3A = sgn(std::max(std::fabs(TMP2A), R(EM20)), TMP2A);
      R TMP1A = DT1V4 * (VZ13 - VZ24) * (VZ13 - VZ24) / TMP3A;
      VX13 = VXl[0] - VXl[2]; VX24 = VXl[1] - VXl[3];
      VX13 = VX13 - TMP1A; VX24 = VX24 + TMP1A;
      R TMP1B = PX2 - PX1;
      R TMP3B = sgn(std::max(std::fabs(TMP1B), R(EM20)), TMP1B);
      R TMP2B = DT1V4 * (VZ13 + VZ24) * (VZ13 + VZ24) / TMP3B;
      VY13 = VYl[0] - VYl[2]; VY24 = VYl[1] - VYl[3];
      VY13 = VY13 + TMP2B; VY24 = VY24 + TMP2B;
    } else if (IHBE == 2 || IHBE == 3) {
      // cdefo3.F:133-172: velocities relative to node 1, warping terms
      R DT1V4 = R(0.5) * DT1;
      R GZX = EXZ / AREA;
      R EXZZ2 = GZX * Z2;
      R EXZ2 = GZX * GZX * DT1V4;
      VXl[2] = VXl[2] - EXZ2 * X3 - VXl[0];
      VXl[1] = VXl[1] + EXZZ2 - EXZ2 * X2 - VXl[0];
      VXl[3] = VXl[3] + EXZZ2 - EXZ2 * X4 - VXl[0];
      VXl[0] = R(0);
      R GZY = EYZ / AREA;
      R EYZZ2 = GZY * Z2;
      R EYZ2 = GZY * GZY * DT1V4;
      VYl[2] = VYl[2] - EYZ2 * Y3 - VYl[0];
      VYl[1] = VYl[1] + EYZZ2 - EYZ2 * Y2 - VYl[0];
      VYl[3] = VYl[3] + EYZZ2 - EYZ2 * Y4 - VYl[0];
      VYl[0] = R(0);
      R ZZZ = (EXZ2 + EYZ2) * Z2;
      VZl[2] = VZl[2] - GZY * Y3 - GZX * X3 - VZl[0];
      VZl[1] = VZl[1] - GZY * Y2 - GZX * X2 - ZZZ - VZl[0];
      VZl[3] = VZl[3] - GZY * Y4 - GZX * X4 - ZZZ - VZl[0];
      VZl[0] = R(0);
      VX13 = -VXl[2]; VX24 = VXl[1] - VXl[3];
      VY13 = -VYl[2]; VY24 = VYl[1] - VYl[3];
    } else {
      // IHBE = 4, cdefo3.F:174-216: z1 = z3 = 0, z4 = z2
      R DT1V4 = R(0.5) * DT1;
      R ZZ2 = R(0.5) * Z2;
      R GZX = EXZ / AREA;
      R EXZZ2 = GZX * ZZ2;
      R EXZ2 = GZX * GZX * DT1V4;
      R EXZ2PY2 = EXZ2 * PY2, EXZ2PY1 = EXZ2 * PY1;
      VXl[0] = VXl[0] - EXZZ2 - EXZ2PY2;
      VXl[2] = VXl[2] - EXZZ2 + EXZ2PY2;
      VXl[1] = VXl[1] + EXZZ2 + EXZ2PY1;
      VXl[3] = VXl[3] + EXZZ2 - EXZ2PY1;
      R GZY = EYZ / AREA;
      R EYZZ2 = GZY * ZZ2;
      R EYZ2 = GZY * GZY * DT1V4;
      R EYZ2PX2 = EYZ2 * PX2, EYZ2PX1 = EYZ2 * PX1;
      VYl[0] = VYl[0] - EYZZ2 + EYZ2PX2;
      VYl[2] = VYl[2] - EYZZ2 - EYZ2PX2;
      VYl[1] = VYl[1] + EYZZ2 - EYZ2PX1;
      VYl[3] = VYl[3] + EYZZ2 + EYZ2PX1;
      VX13 = VXl[0] - VXl[2]; VX24 = VXl[1] - VXl[3];
      VY13 = VYl[0] - VYl[2]; VY24 = VYl[1] - VYl[3];
    }
    EXX = PX1 * VX13 + PX2 * VX24;
    EXY = PY1 * VX13 + PY2 * VX24;
    EXY = EXY + PX1 * VY13 + PX2 * VY24;
    EYY = PY1 * VY13 + PY2 * VY24;
  }
  // CCURV3 (ccurv3.F:61-86)
  R RX[4], RY[4];
  for (int k = 0; k < 4; ++k) {
    RX[k] = E1X * VRL[k][0] + E1Y * VRL[k][1] + E1Z * VRL[k][2];
    RY[k] = E2X * VRL[k][0] + E2Y * VRL[k][1] + E2Z * VRL[k][2];
  }
  R KXX, KYY, KXY;
  {
    R RX13TA = RX[0] - RX[2], RXAVTA = RX[0] + RX[1] + RX[2] + RX[3], RX24TA = RX[1] - RX[3];
    KYY = -PY1 * RX13TA - PY2 * RX24TA;
    KXY = PX1 * RX13TA + PX2 * RX24TA;
    R RY13TA = RY[0] - RY[2], RYAVTA = RY[0] + RY[1] + RY[2] + RY[3], RY24TA = RY[1] - RY[3];
    KXX = PX1 * RY13TA + PX2 * RY24TA;
    KXY = PY1 * RY13TA + PY2 * RY24TA - KXY;
    EXZ = EXZ + RYAVTA * (R(0.25) * AREA);
    EYZ = EYZ - RXAVTA * (R(0.25) * AREA);
  }
  // CSTRA3 (cstra3.F:91-101)
  {
    R FAC1 = DT1 / AREA;
    EXX *= FAC1; EYY *= FAC1; EXY *= FAC1; EYZ *= FAC1; EXZ *= FAC1;
    KXX *= FAC1; KYY *= FAC1; KXY *= FAC1;
  }
  // MULAWC (mulawc.F90:530-560, 596-1100, 2603-2620, 2930-2990)
  R FOR[5] = {0, 0, 0, 0, 0}, MOM[3] = {0, 0, 0};
  R FOR_OLD[5] = {0, 0, 0, 0, 0}, MOM_OLD[3] = {0, 0, 0};
  // GBUF%FOR/MOM of the previous cycle = the stored IP stresses through the weights
  for (int ip = 0; ip < npt; ++ip) {
    R wf = R(WF1[npt - 1][ip]), wm = R(WM1[npt - 1][ip]);
    R s[5];
    for (int c = 0; c < 5; ++c) s[c] = g.sig[(ip * 5 + c) * nel + i];
    for (int c = 0; c < 5; ++c) FOR_OLD[c] = FOR_OLD[c] + wf * s[c];
    for (int c = 0; c < 3; ++c) MOM_OLD[c] = MOM_OLD[c] + wm * s[c];
  }
  for (int c = 0; c < 5; ++c) FOR_OLD[c] *= OFF;
  for (int c = 0; c < 3; ++c) MOM_OLD[c] *= OFF;
  R DEGMB = FOR_OLD[0] * EXX + FOR_OLD[1] * EYY + FOR_OLD[2] * EXY + FOR_OLD[3] * EYZ + FOR_OLD[4] * EXZ;
  R DEGFX = MOM_OLD[0] * KXX + MOM_OLD[1] * KYY + MOM_OLD[2] * KXY;
  R THKN = g.thk[i];
  double wpla = 0;
  // SIGY: EP30 from CCOOR3 (ccoor3.F:126); LAW2 restarts it at 0 and adds each
  // point's yield stress / NPTT (mulawc.F90:565, sigeps02c.F:186-188)
  R SIGY = mt.law == OR_LAW_JOHNSON_COOK ? R(0) : R(1e30);
  for (int ip = 0; ip < npt; ++ip) {
    R THKLY = R(WF1[npt - 1][ip]);
    R THKLYL = THKLY * THK0;
    R WMC = R(WM1[npt - 1][ip]);
    R ZT = R(Z01[npt - 1][ip]) * THK0;
    R DEPSXX = EXX + ZT * KXX, DEPSYY = EYY + ZT * KYY, DEPSXY = EXY + ZT * KXY;
    R DEPSYZ = EYZ, DEPSZX = EXZ;
    R SO[5], SN[5];
    for (int c = 0; c < 5; ++c) SO[c] = g.sig[(ip * 5 + c) * nel + i];
    R EZZ = 0;
    if (mt.law == OR_LAW_ELASTIC) {
      // SIGEPS01C (sigeps01c.F:72-146), ISMSTR/=10
      SN[0] = SO[0] + A11 * DEPSXX + A12 * DEPSYY;
      SN[1] = SO[1] + A12 * DEPSXX + A11 * DEPSYY;
      SN[2] = SO[2] + GG * DEPSXY;
      SN[3] = SO[3] + GS * DEPSYZ;
      SN[4] = SO[4] + GS * DEPSZX;
      EZZ = -NU * (DEPSXX + DEPSYY) / (R(1) - NU);
      THKN = THKN + EZZ * THKLYL * OFF;
    } else {
      // SIGEPS02C -> M2CPLR (m2cplr.F:96-445), IPLA 0/1/2, CC=0, FISOKIN=0, TSTAR=0
      const R CA = g.jca.empty() ? R(mt.jc_a) : g.jca[i];
      const R CB = R(mt.jc_b), CN = R(mt.jc_n), YMAX = R(mt.sigmax);
      const R A1 = YM / (R(1) - NU * NU), A2 = A1 * NU;
      SN[0] = SO[0] + A1 * DEPSXX + A2 * DEPSYY;
      SN[1] = SO[1] + A2 * DEPSXX + A1 * DEPSYY;
      SN[2] = SO[2] + GG * DEPSXY;
      SN[3] = SO[3] + GS * DEPSYZ;
      SN[4] = SO[4] + GS * DEPSZX;
      R PLA = g.pla[ip * nel + i];
      R YLD = (PLA == R(0)) ? CA : CA + CB * std::exp(CN * std::log(PLA));
      YLD = std::min(YLD, YMAX);
      R DPLA = 0;
      const R SMALL = R(1e-7);                       // m2cplr.F:98 SMALL = EM7
      if (pr.ipla == 0) {
        // IPLA = 0 radial return (m2cplr.F:199-230)
        R SVM = std::sqrt(SN[0] * SN[0] + SN[1] * SN[1] - SN[0] * SN[1] + R(3) * SN[2] * SN[2]);
        R RR = std::min(R(1), YLD / (SVM + R(EM15)));
        if (RR < R(1)) {
          SN[0] *= RR; SN[1] *= RR; SN[2] *= RR;
          DPLA = OFF * std::max(R(0), (SVM - YLD) / YM);
          R S1h = R(0.5) * (SN[0] + SN[1]);
          EZZ = DPLA * S1h / YLD;
          PLA = PLA + DPLA;
        }
      } else if (pr.ipla == 1) {
        // IPLA = 1: plane-stress return with NMAX = 3 Newton iterations on DPLA
        // (m2cplr.F:231-378, FISOKIN = 0)
        const R S1 = SN[0] + SN[1], S2 = SN[0] - SN[1], S3 = SN[2];
        const R A = R(0.25) * S1 * S1;
        const R B = R(0.75) * S2 * S2 + R(3) * S3 * S3;
        const R SVM = std::sqrt(A + B);
        if (SVM > YLD && OFF == R(1)) {
          const R NU1 = R(1) / (R(1) - NU), NU2 = R(1) / (R(1) + NU);
          const R H = YLD >= YMAX ? R(0) : CN * CB * std::exp((CN - R(1)) * std::log(PLA + SMALL));
          R DPLA_J = (SVM - YLD) / (R(3) * GG + H);
          const R ANU1 = A * NU1, BNU2 = R(3) * B * NU2, TWOH = R(2) * H;
          R DPLA_I = 0, P = 1, Q = 1, DR = 0;
          for (int it = 0; it < 3; ++it) {
            DPLA_I = DPLA_J;
            const R PLA_I = PLA + DPLA_I;
            DPLA = DPLA_J;
            const R YLD_I = PLA_I == R(0) ? std::min(YMAX, CA) : std::min(YMAX, CA + CB * std::exp(CN * std::log(PLA_I)));
            DR = R(0.5) * YM * DPLA_I / YLD_I;
            P = R(1) / (R(1) + DR * NU1);
            Q = R(1) / (R(1) + R(3) * DR * NU2);
            const R P2 = P * P, Q2 = Q * Q;
            const R F = A * P2 + B * Q2 - YLD_I * YLD_I;
            const R DF = -(ANU1 * P2 * P + BNU2 * Q2 * Q) * (YM - DR * TWOH) / YLD_I - TWOH * YLD_I;
            DPLA_J = DPLA_I > R(0) ? std::max(R(0), DPLA_I - F / DF) : R(0);
          }
          PLA = PLA + DPLA_I;
          const R T1 = (SN[0] + SN[1]) * P, T2 = (SN[0] - SN[1]) * Q;
          SN[0] = R(0.5) * (T1 + T2);
          SN[1] = R(0.5) * (T1 - T2);
          SN[2] = SN[2] * Q;
          EZZ = DR * T1 / YM;
        }
      } else {
        // IPLA = 2: approximate normal projection, then radial return (m2cplr.F:379-445)
        const R SVM2 = SN[0] * SN[0] + SN[1] * SN[1] - SN[0] * SN[1] + R(3) * SN[2] * SN[2];
        R SVM = std::sqrt(SVM2);
        const R YLD2 = YLD * YLD;
        if (SVM2 > YLD2 && OFF == R(1)) {
          const R H = YLD >= YMAX ? R(0) : CN * CB * std::exp((CN - R(1)) * std::log(PLA + SMALL));
          const R AA = (SVM2 - YLD2) / (R(5) * SVM2 + R(3) * (-SN[0] * SN[1] + SN[2] * SN[2]));
          const R S1 = (R(1) - R(2) * AA) * SN[0] + AA * SN[1];
          const R S2 = AA * SN[0] + (R(1) - R(2) * AA) * SN[1];
          const R S3 = (R(1) - R(3) * AA) * SN[2];
          SN[0] = S1; SN[1] = S2; SN[2] = S3;
          DPLA = OFF * (SVM - YLD) / (R(3) * GG + H);
          PLA = PLA + DPLA;
          YLD = YLD + H * DPLA;
          SVM = std::sqrt(SN[0] * SN[0] + SN[1] * SN[1] - SN[0] * SN[1] + R(3) * SN[2] * SN[2]);
          const R RR = std::min(R(1), YLD / std::max(R(EM20), SVM));
          SN[0] *= RR; SN[1] *= RR; SN[2] *= RR;
          EZZ = DPLA * R(0.5) * (SN[0] + SN[1]) / YLD;
        }
      }
      g.pla[ip * nel + i] = PLA;
      SIGY = SIGY + YLD / R(npt);
      // sigeps02c.F:215-224
      EZZ = -(DEPSXX + DEPSYY) * NU - (R(1) - R(2) * NU) * EZZ;
      EZZ = EZZ / (R(1) - NU);
      THKN = THKN + EZZ * THKLYL * OFF;
      wpla += double(YLD) * double(DPLA) * double(AREA) * double(THKLYL);
    }
    for (int c = 0; c < 5; ++c) g.sig[(ip * 5 + c) * nel + i] = SN[c];
    for (int c = 0; c < 5; ++c) FOR[c] = FOR[c] + THKLY * SN[c];
    for (int c = 0; c < 3; ++c) MOM[c] = MOM[c] + WMC * SN[c];
  }
  wpla_out += wpla;
  g.thk[i] = std::max(THKN, R(EM30));
  for (int c = 0; c < 5; ++c) FOR[c] *= OFF;
  for (int c = 0; c < 3; ++c) MOM[c] *= OFF;
  DEGMB = DEGMB + FOR[0] * EXX + FOR[1] * EYY + FOR[2] * EXY + FOR[3] * EYZ + FOR[4] * EXZ;
  DEGFX = DEGFX + MOM[0] * KXX + MOM[1] * KYY + MOM[2] * KXY;
  {
    R VOL2 = R(0.5) * VOL0;
    g.eint[0 * nel + i] = g.eint[0 * nel + i] + DEGMB * VOL2;
    g.eint[1 * nel + i] = g.eint[1 * nel + i] + DEGFX * THK0 * VOL2;
  }
  // Hourglass forces (cforc3.F:593-640): MHVIS3 for one integration point,
  // CHSTI3 for IHBE = 2, CHVIS3 otherwise; ISMSTR=2, NODADT=0, HELAS=HVISC=1/2,
  // HVLIN=0.  H1j/H2j/H3j: membrane x, y and bending hourglass forces of corners
  // 1..3 (corner 4 follows from their sum being zero), B1j/B2j the moments.
  R H1j[3], H2j[3], H3j[3], B1j[4], B2j[4];
  {
    const R HELAS = R(0.5), HVISC = R(0.5);
    R GAMA[4];
    if (IHBE >= 1) {
      R PX1V = PX1 * VHX, PX2V = PX2 * VHX, PY1V = PY1 * VHY, PY2V = PY2 * VHY;
      GAMA[0] = OFF * (R(1) - PX1V - PY1V);
      GAMA[2] = OFF * (R(1) + PX1V + PY1V);
      GAMA[1] = OFF * (-R(1) - PX2V - PY2V);
      GAMA[3] = OFF * (-R(1) + PX2V + PY2V);
    } else {
      GAMA[0] = OFF; GAMA[2] = OFF; GAMA[1] = -OFF; GAMA[3] = -OFF;
    }
    const bool degen = nc[2] == nc[3];
    R* HOUR = &g.hourg[0];
    R EHOU;
    if (npt == 1) {
      // MHVIS3 (mhvis3.F:109-363): elastic membrane and bending terms, V-shape
      // bending damping Dn, no hourglass moments
      const R H4 = R(pr.dn);
      R FAC = R(0.25) * RHO * THK0;
      R H1L = R(0), H1Q = R(0), H2L = R(0), H2Q = R(0);
      R H4L = FAC * std::sqrt(HVISC * H4 * AREA);
      R H4Q = std::sqrt(HVISC * H4) * H4L * R(100);
      H4L = H4L * SSP;
      FAC = R(0.25) * YM * THK0 * DT1 * HELAS;
      R H1e = H1 * FAC, H2e = H2 * FAC;
      if (degen) { H1Q = H1L = H2Q = H2L = H4L = H4Q = H1e = H2e = R(0); }
      R Hm1[4], Hm2[4], Hb[4];
      R HG1, HG2;
      if (IHBE < 1) {
        HG1 = VXl[0] - VXl[1] + VXl[2] - VXl[3];
        HG2 = VYl[0] - VYl[1] + VYl[2] - VYl[3];
      } else {
        HG1 = VXl[0] * GAMA[0] + VXl[1] * GAMA[1] + VXl[2] * GAMA[2] + VXl[3] * GAMA[3];
        HG2 = VYl[0] * GAMA[0] + VYl[1] * GAMA[1] + VYl[2] * GAMA[2] + VYl[3] * GAMA[3];
      }
      R hour1 = HOUR[0 * nel + i] + HG1 * H1e;
      R hour2 = HOUR[1 * nel + i] + HG2 * H1e;
      HG1 = HG1 * (H1L + H1Q * std::fabs(HG1));
      HG2 = HG2 * (H1L + H1Q * std::fabs(HG2));
      if (IHBE < 1) {
        Hm1[0] = hour1 + HG1; Hm1[1] = -hour1 - HG1; Hm1[2] = hour1 + HG1; Hm1[3] = -hour1 - HG1;
        Hm2[0] = hour2 + HG2; Hm2[1] = -hour2 - HG2; Hm2[2] = hour2 + HG2; Hm2[3] = -hour2 - HG2;
      } else {
        for (int k = 0; k < 4; ++k) { Hm1[k] = (hour1 + HG1) * GAMA[k]; Hm2[k] = (hour2 + HG2) * GAMA[k]; }
      }
      EHOU = VXl[0] * Hm1[0] + VXl[1] * Hm1[1] + VXl[2] * Hm1[2] + VXl[3] * Hm1[3] +
             VYl[0] * Hm2[0] + VYl[1] * Hm2[1] + VYl[2] * Hm2[2] + VYl[3] * Hm2[3];
      if (IHBE < 1) HG1 = VZl[0] - VZl[1] + VZl[2] - VZl[3];
      else HG1 = VZl[0] * GAMA[0] + VZl[1] * GAMA[1] + VZl[2] * GAMA[2] + VZl[3] * GAMA[3];
      R hour3 = HOUR[2 * nel + i] + HG1 * H2e;
      HG1 = HG1 * (H2L + H2Q * std::fabs(HG1));
      if (IHBE < 1) {
        Hb[0] = hour3 + HG1; Hb[1] = -hour3 - HG1; Hb[2] = hour3 + HG1; Hb[3] = -hour3 - HG1;
      } else {
        for (int k = 0; k < 4; ++k) Hb[k] = (hour3 + HG1) * GAMA[k];
      }
      HG1 = VZl[0] + VZl[1] - VZl[2] - VZl[3];
      HG1 = HG1 * (H4L + H4Q * std::fabs(HG1));
      Hb[0] = Hb[0] + HG1; Hb[1] = Hb[1] + HG1; Hb[2] = Hb[2] - HG1; Hb[3] = Hb[3] - HG1;
      HG1 = VZl[0] - VZl[1] - VZl[2] + VZl[3];
      HG1 = HG1 * (H4L + H4Q * std::fabs(HG1));
      Hb[0] = Hb[0] + HG1; Hb[1] = Hb[1] - HG1; Hb[2] = Hb[2] - HG1; Hb[3] = Hb[3] + HG1;
      for (int k = 0; k < 3; ++k) { H1j[k] = Hm1[k]; H2j[k] = Hm2[k]; H3j[k] = Hb[k]; }
      for (int k = 0; k < 4; ++k) { B1j[k] = R(0); B2j[k] = R(0); }
      EHOU = EHOU + VZl[0] * Hb[0] + VZl[1] * Hb[1] + VZl[2] * Hb[2] + VZl[3] * Hb[3];
      EHOU = DT1 * EHOU;
      HOUR[0 * nel + i] = hour1; HOUR[1 * nel + i] = hour2; HOUR[2 * nel + i] = hour3;
    } else if (IHBE == 2) {
      // CHSTI3 (chsti3.F:119-320): elastic hourglass stiffness bounded by the
      // yield stress SIGY, viscous rotational terms with SRH3 = sqrt(hr)
      // (resol_init.F:676-682)
      const R HP1 = H1, HP2 = H2, H3s = R(std::sqrt(pr.hr));
      const R SHFPR3 = SHF / (R(3) * (R(1) + NU));
      R FAC = R(0.25) * RHO * THK02;
      R H3L = H3s * R(0.072169) * FAC * AREA;
      R H3Q = H3s * H3L * R(100);
      H3L = H3L * SSP;
      FAC = YM * THK0 * DT1 * R(0.125);
      R H1e = HP1 * FAC;
      const R B1 = PX1 * PX1 + PY1 * PY1, B2 = PX2 * PX2 + PY2 * PY2;
      R H2e = HP2 * FAC * THK02 * SHFPR3 / (B1 + B2);
      if (degen) { H3Q = H3L = H1e = H2e = R(0); }
      R HG1 = VXl[0] * GAMA[0] + VXl[1] * GAMA[1] + VXl[2] * GAMA[2] + VXl[3] * GAMA[3];
      R HG2 = VYl[0] * GAMA[0] + VYl[1] * GAMA[1] + VYl[2] * GAMA[2] + VYl[3] * GAMA[3];
      R hour1 = HOUR[0 * nel + i] + HG1 * H1e;
      R hour2 = HOUR[1 * nel + i] + HG2 * H1e;
      R FMAX = R(0.5) * SIGY * THK0 * std::sqrt(AREA) * HP1;
      hour1 = sgn(std::min(std::fabs(hour1), FMAX), hour1);
      hour2 = sgn(std::min(std::fabs(hour2), FMAX), hour2);
      for (int k = 0; k < 3; ++k) { H1j[k] = hour1 * GAMA[k]; H2j[k] = hour2 * GAMA[k]; }
      EHOU = hour1 * HG1 + hour2 * HG2;
      HG1 = VZl[0] * GAMA[0] + VZl[1] * GAMA[1] + VZl[2] * GAMA[2] + VZl[3] * GAMA[3];
      R hour3 = HOUR[2 * nel + i] + HG1 * H2e;
      FMAX = R(0.25) * SIGY * THK0 * THK0 * HP2;
      hour3 = sgn(std::min(std::fabs(hour3), FMAX), hour3);
      for (int k = 0; k < 3; ++k) H3j[k] = hour3 * GAMA[k];
      EHOU = EHOU + hour3 * HG1;
      HG1 = RX[0] - RX[1] + RX[2] - RX[3];
      HG2 = RY[0] - RY[1] + RY[2] - RY[3];
      R HOUR4 = HG1 * (H3L + H3Q * std::fabs(HG1));
      R HOUR5 = HG2 * (H3L + H3Q * std::fabs(HG2));
      EHOU = EHOU + HOUR4 * HG1 + HOUR5 * HG2;
      EHOU = DT1 * EHOU * OFF;
      B1j[0] = HOUR4 * OFF; B1j[1] = -HOUR4 * OFF; B1j[2] = HOUR4 * OFF; B1j[3] = -HOUR4 * OFF;
      B2j[0] = HOUR5 * OFF; B2j[1] = -HOUR5 * OFF; B2j[2] = HOUR5 * OFF; B2j[3] = -HOUR5 * OFF;
      HOUR[0 * nel + i] = hour1; HOUR[1 * nel + i] = hour2; HOUR[2 * nel + i] = hour3;
    } else {
      // CHVIS3 (chvis3.F:116-300)
      const R HVLIN = R(0);
      R SHFPR3 = SHF / (R(3) * (R(1) + NU));
      R HVISH1 = HVISC * H1, HVISH2 = HVISC * H2;
      R R0 = R(0.25) * RHO;
      R R1 = R0 * R(100);
      R0 = R0 * HVLIN;
      R A1c = R1 * HVISH1;
      R SRSHFPR3 = std::sqrt(SHFPR3);
      R A3c = R1 * HVISH2 * SRSHFPR3;
      R A5c = HELAS * H3 * R1 * R(0.072169);
      R R0e = R(0.25) * YM * HELAS;
      R A7c = H1 * R0e;
      R A8c = H2 * R0e * SHFPR3;
      R T2A = THK02 * AREA;
      R TSA = std::sqrt(T2A);
      R H1Q = A1c * TSA, H1L = R(0);
      R H2Q = A3c * THK02, H2L = R(0);
      R H3Q = A5c * T2A, H3L = R(0);
      (void)R0;
      R TD = THK0 * DT1;
      R HH1 = A7c * TD;
      R B1 = PX1 * PX1 + PY1 * PY1, B2 = PX2 * PX2 + PY2 * PY2;
      R HH2 = A8c * THK02 * TD / (B1 + B2);
      if (degen) { H1Q = H1L = H2Q = H2L = H3Q = H3L = HH1 = HH2 = R(0); }
      R HG1, HG2;
      if (IHBE < 1) {
        HG1 = (VXl[0] - VXl[1] + VXl[2] - VXl[3]) * OFF;
        HG2 = (VYl[0] - VYl[1] + VYl[2] - VYl[3]) * OFF;
      } else {
        HG1 = VXl[0] * GAMA[0] + VXl[1] * GAMA[1] + VXl[2] * GAMA[2] + VXl[3] * GAMA[3];
        HG2 = VYl[0] * GAMA[0] + VYl[1] * GAMA[1] + VYl[2] * GAMA[2] + VYl[3] * GAMA[3];
      }
      R hour1 = HOUR[0 * nel + i] + HG1 * HH1;
      R hour2 = HOUR[1 * nel + i] + HG2 * HH1;
      R HOUR1A = hour1 + HG1 * (H1L + H1Q * std::fabs(HG1));
      R HOUR2A = hour2 + HG2 * (H1L + H1Q * std::fabs(HG2));
      for (int k = 0; k < 3; ++k) { H1j[k] = HOUR1A * GAMA[k]; H2j[k] = HOUR2A * GAMA[k]; }
      EHOU = HOUR1A * HG1 + HOUR2A * HG2;
      if (IHBE < 1) HG1 = (VZl[0] - VZl[1] + VZl[2] - VZl[3]) * OFF;
      else HG1 = VZl[0] * GAMA[0] + VZl[1] * GAMA[1] + VZl[2] * GAMA[2] + VZl[3] * GAMA[3];
      R hour3 = HOUR[2 * nel + i] + HG1 * HH2;
      R HOUR3A = hour3 + HG1 * (H2L + H2Q * std::fabs(HG1));
      for (int k = 0; k < 3; ++k) H3j[k] = HOUR3A * GAMA[k];
      EHOU = EHOU + HOUR3A * HG1;
      HG1 = RX[0] - RX[1] + RX[2] - RX[3];
      HG2 = RY[0] - RY[1] + RY[2] - RY[3];
      R HOUR4 = HG1 * (H3L + H3Q * std::fabs(HG1));
      R HOUR5 = HG2 * (H3L + H3Q * std::fabs(HG2));
      EHOU = EHOU + HOUR4 * HG1 + HOUR5 * HG2;
      EHOU = DT1 * EHOU * OFF;
      B1j[0] = HOUR4 * OFF; B1j[1] = -HOUR4 * OFF; B1j[2] = HOUR4 * OFF; B1j[3] = -HOUR4 * OFF;
      B2j[0] = HOUR5 * OFF; B2j[1] = -HOUR5 * OFF; B2j[2] = HOUR5 * OFF; B2j[3] = -HOUR5 * OFF;
      HOUR[0 * nel + i] = hour1; HOUR[1 * nel + i] = hour2; HOUR[2 * nel + i] = hour3;
    }
    ehou_out += double(EHOU);
  }
  // CDT3 (cdt3.F:110-115, 203-214), NODADT=0, IDTMIN(3)=2
  {
    R DT = R(m.cfg.dtfac_shell) * ALDT / SSP;
    if (double(DT) <= m.cfg.dtmin_shell) return OR_E_DTMIN;
    dt2t_out = std::min(dt2t_out, double(DT));
  }
  // CFINT3 (cfint3.F:173-260), ISIGI=0
  R Fg[3][4], Mg[3][4];
  {
    R F1A = FOR[0] * THK0, F2A = FOR[1] * THK0, F3A = FOR[2] * THK0, F4A = FOR[3] * THK0, F5A = FOR[4] * THK0;
    R M4 = F4A * AREA, M5 = F5A * AREA;
    R F12 = F1A * PX2 + F3A * PY2, F22 = F2A * PY2 + F3A * PX2, F32 = F5A * PX2 + F4A * PY2;
    R F11 = F1A * PX1 + F3A * PY1, F21 = F2A * PY1 + F3A * PX1, F31 = F5A * PX1 + F4A * PY1;
    R G11 = F11 + H1j[0], G13 = H1j[2] - F11, G21 = F21 + H2j[0], G23 = H2j[2] - F21;
    R G31 = F31 + H3j[0], G33 = H3j[2] - F31;
    R G12 = F12 + H1j[1], G22 = F22 + H2j[1], G32 = F32 + H3j[1];
    R Gc[3][3] = {{G11, G12, G13}, {G21, G22, G23}, {G31, G32, G33}};
    for (int k = 0; k < 3; ++k) {
      Fg[0][k] = E1X * Gc[0][k] + E2X * Gc[1][k] + E3X * Gc[2][k];
      Fg[1][k] = E1Y * Gc[0][k] + E2Y * Gc[1][k] + E3Y * Gc[2][k];
      Fg[2][k] = E1Z * Gc[0][k] + E2Z * Gc[1][k] + E3Z * Gc[2][k];
    }
    for (int c = 0; c < 3; ++c) Fg[c][3] = -Fg[c][0] - Fg[c][1] - Fg[c][2];
    if (IHBE >= 2 && npt != 1) {          // cfint3.F:208-214, warping moments
      M4 = M4 + (H2j[0] + H2j[2]) * Z2;
      M5 = M5 + (H1j[0] + H1j[2]) * Z2;
    }
    R M1A = MOM[0] * THK02, M2A = MOM[1] * THK02, M3A = MOM[2] * THK02;
    M4 = M4 * R(0.25); M5 = M5 * R(0.25);
    R M11 = -M2A * PY1 - M3A * PX1, M21 = M1A * PX1 + M3A * PY1;
    R M12 = -M2A * PY2 - M3A * PX2, M22 = M1A * PX2 + M3A * PY2;
    R Gm1[4] = {M11 - M4 + B1j[0], M12 - M4 + B1j[1], -M11 - M4 + B1j[2], -M12 - M4 + B1j[3]};
    R Gm2[4] = {M21 + M5 + B2j[0], M22 + M5 + B2j[1], -M21 + M5 + B2j[2], -M22 + M5 + B2j[3]};
    for (int k = 0; k < 4; ++k) {
      Mg[0][k] = E1X * Gm1[k] + E2X * Gm2[k];
      Mg[1][k] = E1Y * Gm1[k] + E2Y * Gm2[k];
      Mg[2][k] = E1Z * Gm1[k] + E2Z * Gm2[k];
    }
  }
  // /PLOAD-style uniform pressure (load_pressure.F:201-207): F = -p N/8 per node,
  // N = (x3-x1) x (x4-x2) from the current coordinates, added to the corner slot;
  // the diagonals in FP64 (my_real X differences in the FP64 form), the cross
  // product in my_real.
  R PF[3] = {0, 0, 0};
  if (pr.pressure != 0.0) {
    double ax = XG[2] - XG[0], ay = YG[2] - YG[0], az = ZG[2] - ZG[0];
    double bx = XG[3] - XG[1], by = YG[3] - YG[1], bz = ZG[3] - ZG[1];
    if (!split) { ax = P.x[3*nc[2]] - P.x[3*nc[0]]; ay = P.x[3*nc[2]+1] - P.x[3*nc[0]+1]; az = P.x[3*nc[2]+2] - P.x[3*nc[0]+2];
                  bx = P.x[3*nc[3]] - P.x[3*nc[1]]; by = P.x[3*nc[3]+1] - P.x[3*nc[1]+1]; bz = P.x[3*nc[3]+2] - P.x[3*nc[1]+2]; }
    const R Ax = R(ax), Ay = R(ay), Az = R(az), Bx = R(bx), By = R(by), Bz = R(bz);
    R NX = Ay * Bz - Az * By, NY = Az * Bx - Ax * Bz, NZ = Ax * By - Ay * Bx;
    R AA = -R(pr.pressure) * R(0.125);
    PF[0] = AA * NX; PF[1] = AA * NY; PF[2] = AA * NZ;
  }
  // CUPDT3P (cupdt3.F:1040-1063): FSKY = -F, -M
  for (int k = 0; k < 4; ++k) {
    long s = g.iadc[4 * i + k];
    R* f = &P.fsky[8 * s];
    f[0] = -Fg[0][k] + PF[0]; f[1] = -Fg[1][k] + PF[1]; f[2] = -Fg[2][k] + PF[2];
    f[3] = -Mg[0][k]; f[4] = -Mg[1][k]; f[5] = -Mg[2][k];
    f[6] = 0; f[7] = 0;
  }
  return OR_OK;
}

// ----------------------------------------------------------------------------
// FINTER (tools/curve/finter.F): first segment whose right end is >= XX (the
// last one beyond the end), linear inside and beyond both ends, evaluated from
// the nearer end of the segment; a one-point function is constant.
// ----------------------------------------------------------------------------
template <class R>
R finter(const Func& f, R XX) {
  const int n = (int)f.x.size();
  if (n == 1) return R(f.y[0]);
  R DX2 = R(f.x[0]) - XX;
  for (int i = 1; i < n; ++i) {
    const R DX1 = -DX2;
    DX2 = R(f.x[i]) - XX;
    if (DX2 >= R(0) || i == n - 1) {
      const R DIV0 = R(f.x[i]) - R(f.x[i - 1]);
      R DIV = std::max(std::fabs(DIV0), R(1e-16));
      DIV = sgn(DIV, DIV0);
      const R DERI = (R(f.y[i]) - R(f.y[i - 1])) / DIV;
      return DX1 <= DX2 ? R(f.y[i - 1]) + DX1 * DERI : R(f.y[i]) - DX2 * DERI;
    }
  }
  return R(0);
}

// BCS1V (bcs1.F): zero the components of a (or v) along the fixed directions of
// code lcod (4 = x, 2 = y, 1 = z) of the global axes (sk == null) or of skew sk
// (rows x', y', z'), projecting them out in the reference's order.
template <class R>
void bcs1v(int lcod, const double* sk, R* a) {
  if (!lcod) return;
  if (!sk) {
    if (lcod & 4) a[0] = R(0);
    if (lcod & 2) a[1] = R(0);
    if (lcod & 1) a[2] = R(0);
    return;
  }
  if (lcod == 7) { a[0] = a[1] = a[2] = R(0); return; }
  auto proj = [&](int r) {
    const R s0 = R(sk[3 * r]), s1 = R(sk[3 * r + 1]), s2 = R(sk[3 * r + 2]);
    const R AA = s0 * a[0] + s1 * a[1] + s2 * a[2];
    a[0] = a[0] - s0 * AA; a[1] = a[1] - s1 * AA; a[2] = a[2] - s2 * AA;
  };
  switch (lcod) {
    case 1: proj(2); break;
    case 2: proj(1); break;
    case 3: proj(2); proj(1); break;
    case 4: proj(0); break;
    case 5: proj(2); proj(0); break;
    case 6: proj(0); proj(1); break;
  }
}

// FORCE (force.F90, Parith/ON): load slots at the start of the cycle, at TT and
// the coordinates of the cycle's start.  Returns the concentrated loads' power
// sum 1/2 (F(TT-DT1)+F(TT)).v (WFEXC) and adds the segments' DT1 F.sum v to wext.
template <class R>
double load_pass(Model<R>& m, int p, double tt, double dt1, double& wext) {
  PartData<R>& P = m.parts[p];
  double wfexc = 0;
  for (auto& c : m.cloads) {
    if (c.part != p) continue;
    const Func& f = m.funcs[c.func];
    const R ts = R(tt);
    const R a0 = R(c.fcy) * finter<R>(f, (ts - R(dt1)) * R(c.fcx));
    const R aa = R(c.fcy) * finter<R>(f, ts * R(c.fcx));
    R* fs = &P.fsky[8 * c.slot];
    for (int k = 0; k < 8; ++k) fs[k] = R(0);
    const bool rot = c.dir > 3;
    const int d = rot ? c.dir - 4 : c.dir - 1;
    const R* vel = rot ? &P.vr[3 * c.node] : &P.v[3 * c.node];
    R vv;
    if (c.skew < 0) {
      fs[(rot ? 3 : 0) + d] = aa;
      vv = vel[d];
    } else {
      const double* sk = m.skews[c.skew].data() + 3 * d;
      vv = R(sk[0]) * vel[0] + R(sk[1]) * vel[1] + R(sk[2]) * vel[2];
      for (int k = 0; k < 3; ++k) fs[(rot ? 3 : 0) + k] = R(sk[k]) * aa;
    }
    wfexc += double(R(0.5) * (a0 + aa) * vv);
  }
  for (auto& q : m.ploads) {
    if (q.part != p) continue;
    const R aa = R(q.fcy) * finter<R>(m.funcs[q.func], R(tt) * R(q.fcx));
    auto X = [&](int k, int c) { return R(P.x[3 * q.n[k] + c]); };
    const bool quad = q.n[3] >= 0;
    const int k4 = quad ? 3 : 2;          // triangle: (x3 - x1) x (x3 - x2) / 6
    const int k2 = 1;
    const R ax = X(2, 0) - X(0, 0), ay = X(2, 1) - X(0, 1), az = X(2, 2) - X(0, 2);
    const R bx = X(k4, 0) - X(k2, 0), by = X(k4, 1) - X(k2, 1), bz = X(k4, 2) - X(k2, 2);
    const R NX = ay * bz - az * by, NY = az * bx - ax * bz, NZ = ax * by - ay * bx;
    const R c = quad ? R(0.125) : R(1.0 / 6.0);
    const R fx = aa * NX * c, fy = aa * NY * c, fz = aa * NZ * c;
    R sv[3] = {0, 0, 0};
    for (int k = 0; k < (quad ? 4 : 3); ++k) {
      R* fs = &P.fsky[8 * q.slot[k]];
      for (int j = 0; j < 8; ++j) fs[j] = R(0);
      fs[0] = fx; fs[1] = fy; fs[2] = fz;
      for (int j = 0; j < 3; ++j) sv[j] = sv[j] + P.v[3 * q.n[k] + j];
    }
    wext += double(R(dt1) * (fx * sv[0] + fy * sv[1] + fz * sv[2]));
  }
  return wfexc;
}

// ----------------------------------------------------------------------------
// One cycle of one part: element pass, ASSPAR4, dt, ACCELE, BCS10, VELOCITY, DEPLA.
// ----------------------------------------------------------------------------
// ROTBMR (engine/source/tools/skew/rotbmr.F): turns the principal frame RBY(1:9)
// by the rotation vector DT*VR (VR in the principal frame), then re-orthonormalises
template <class R>
void rotbmr(const R* vr, R* rby, R dt) {
  const R rx = dt * vr[0], ry = dt * vr[1], rz = dt * vr[2];
  const R rx2 = rx * rx, ry2 = ry * ry, rz2 = rz * rz;
  const R r2 = std::max(R(1e-10), rx2 + ry2 + rz2);
  const R r = std::sqrt(r2);
  R c = std::cos(r);
  const R cm1 = R(1) - c;
  c = c * r2;
  const R s = std::sin(r) * r;
  const R sz = rz * s, cz = rz * cm1;
  const R e11 = rx2 * cm1 + c, e22 = ry2 * cm1 + c;
  R e12 = rx * ry * cm1;
  const R e21 = e12 - sz;
  e12 = e12 + sz;
  const R e13 = rx * cz - ry * s, e23 = ry * cz + rx * s;
  R b11 = rby[0] * e11 + rby[3] * e12 + rby[6] * e13;
  R b21 = rby[1] * e11 + rby[4] * e12 + rby[7] * e13;
  R b31 = rby[2] * e11 + rby[5] * e12 + rby[8] * e13;
  R b12 = rby[0] * e21 + rby[3] * e22 + rby[6] * e23;
  R b22 = rby[1] * e21 + rby[4] * e22 + rby[7] * e23;
  R b32 = rby[2] * e21 + rby[5] * e22 + rby[8] * e23;
  R bn = std::sqrt(b11 * b11 + b21 * b21 + b31 * b31);
  b11 = b11 / bn; b21 = b21 / bn; b31 = b31 / bn;
  bn = std::sqrt(b12 * b12 + b22 * b22 + b32 * b32);
  b12 = b12 / bn; b22 = b22 / bn; b32 = b32 / bn;
  rby[0] = b11; rby[1] = b21; rby[2] = b31;
  rby[3] = b12; rby[4] = b22; rby[5] = b32;
  rby[6] = b21 * b32 - b31 * b22;
  rby[7] = b31 * b12 - b11 * b32;
  rby[8] = b11 * b22 - b21 * b12;
}

// RBYFOR -> RGBODFP for one rigid body (rgbodfp.F, explicit 3D, no rotational BCS on
// the main node, Ispher 2): the secondary nodes' forces, and their moments about
// the main node, summed in DOUBLE PRECISION (the reference's RBF6 six-part exact
// sum; here in the secondary-node order) onto the main node (phase 1 and 2); the
// principal frame turned by the main node's rotational velocity over DT1; the
// moment expressed in the principal frame, the gyroscopic terms added (Euler's
// equations), and replaced by the pseudo moment IN(M) * rotational acceleration
// (IN(M) = the smallest principal inertia) so that ACCELE's AR = AM / IN(M) is the
// body's rotational acceleration.  af, am: the main node's force and moment sums
// (ASSPAR4), updated.
template <class R, class SUM>
void rgbodfp(RBody<R>& rb, const PartData<R>& P, R* af, R* am, R dt1, SUM raw) {
  const int M = rb.master;
  R* rby = rb.rby;
  const R inm = P.in[M];
  rby[9] = std::max(rby[9], inm);
  rby[10] = std::max(rby[10], inm);
  rby[11] = std::max(rby[11], inm);
  double S[6] = {0, 0, 0, 0, 0, 0};
  for (int n : rb.slaves) {
    R f[3], mo[3];
    raw(n, f, mo);
    const R dx = R(P.x[3 * n] - P.x[3 * M]), dy = R(P.x[3 * n + 1] - P.x[3 * M + 1]),
            dz = R(P.x[3 * n + 2] - P.x[3 * M + 2]);
    const R f6 = mo[0] + dy * f[2] - dz * f[1];
    const R f7 = mo[1] + dz * f[0] - dx * f[2];
    const R f8 = mo[2] + dx * f[1] - dy * f[0];
    S[0] += double(f[0]); S[1] += double(f[1]); S[2] += double(f[2]);
    S[3] += double(f6); S[4] += double(f7); S[5] += double(f8);
  }
  for (int c = 0; c < 3; ++c) { af[c] = R(double(af[c]) + S[c]); am[c] = R(double(am[c]) + S[3 + c]); }
  const R* vr = &P.vr[3 * M];
  const R wa1 = am[0], wa2 = am[1], wa3 = am[2];
  R vi[3];
  vi[0] = rby[0] * vr[0] + rby[1] * vr[1] + rby[2] * vr[2];
  vi[1] = rby[3] * vr[0] + rby[4] * vr[1] + rby[5] * vr[2];
  vi[2] = rby[6] * vr[0] + rby[7] * vr[1] + rby[8] * vr[2];
  rotbmr(vi, rby, dt1);
  R p1 = rby[0] * wa1 + rby[1] * wa2 + rby[2] * wa3;
  R p2 = rby[3] * wa1 + rby[4] * wa2 + rby[5] * wa3;
  R p3 = rby[6] * wa1 + rby[7] * wa2 + rby[8] * wa3;
  p1 = p1 + (rby[10] - rby[11]) * vi[1] * vi[2];
  p2 = p2 + (rby[11] - rby[9]) * vi[2] * vi[0];
  p3 = p3 + (rby[9] - rby[10]) * vi[0] * vi[1];
  const R q1 = p1 * inm / rby[9], q2 = p2 * inm / rby[10], q3 = p3 * inm / rby[11];
  am[0] = rby[0] * q1 + rby[3] * q2 + rby[6] * q3;
  am[1] = rby[1] * q1 + rby[4] * q2 + rby[7] * q3;
  am[2] = rby[2] * q1 + rby[5] * q2 + rby[8] * q3;
}

template <class R>
int cycle(Model<R>& m, int p, or_ecycle_time& t, int nthreads, bool last) {
  PartData<R>& P = m.parts[p];
  // RESOL :2639-2640
  t.dt1 = t.dt2;
  const double DT1 = t.dt1;
  double dt2t = 1e6;   // EP06
  int status = OR_OK;
  int eidx = -1;
  int ityp = 0, nelt = -1;
  double ehou = 0, wpla = 0;
  // FORCE (resol.F:2847): load slots, before the element pass
  double wext_seg = 0;
  const double wfexc = load_pass(m, p, t.tt, DT1, wext_seg);
  // shells first (FORINTC :4012), then solids (FORINT :4096)
  for (auto& g : m.shell) {
    if (g.part != p) continue;
    std::vector<double> dtl(g.nel, 1e30), eh(g.nel, 0), wp(g.nel, 0);
    std::vector<int> st(g.nel, 0);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < g.nel; ++i) {
      double d = 1e30, e = 0, w = 0;
      st[i] = shell_element(m, g, P, i, DT1, d, e, w);
      dtl[i] = d; eh[i] = e; wp[i] = w;
    }
    for (int i = 0; i < g.nel; ++i) {
      if (st[i] && !status) { status = st[i]; eidx = g.gofs + i; }
      ehou += eh[i]; wpla += wp[i];
      if (dtl[i] < dt2t) { dt2t = dtl[i]; ityp = 3; nelt = g.gofs + i; }
    }
  }
  for (auto& g : m.hex) {
    if (g.part != p) continue;
    std::vector<double> dtl(g.nel, 1e30), eh(g.nel, 0), wp(g.nel, 0);
    std::vector<int> st(g.nel, 0);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < g.nel; ++i) {
      double d = 1e30, e = 0, w = 0;
      st[i] = hex_element(m, g, P, i, DT1, d, e, w);
      dtl[i] = d; eh[i] = e; wp[i] = w;
    }
    for (int i = 0; i < g.nel; ++i) {
      if (st[i] && !status) { status = st[i]; eidx = g.gofs + i; }
      ehou += eh[i]; wpla += wp[i];
      if (dtl[i] < dt2t) { dt2t = dtl[i]; ityp = 1; nelt = g.gofs + i; }
    }
  }
  if (status) { m.errcode = status; m.errindex = eidx; return status; }
  P.ehour += ehou;
  P.wplast += wpla;
  // dt logic (resol.F:5853-5858, 6080, 6224-6226)
  double DT2 = 1e6;
  if (dt2t < DT2) { DT2 = dt2t; t.ityptst = ityp; t.neltst = nelt; }
  DT2 = std::min(std::min(DT2, m.cfg.dt_growth * t.dt2old), m.cfg.dtmx);
  if (m.cfg.precision == OR_PREC_SPLIT) DT2 = double(float(DT2));
  t.dt2 = DT2;
  t.dt2old = DT2;
  t.dt12 = 0.5 * (t.dt1 + t.dt2);
  // external work: segments with DT1 in FORCE, concentrated loads WFEXC*DT2 (resol.F:6238)
  P.wext += wext_seg;
  P.wext += wfexc * DT2;
  const R DT12 = R(t.dt12);
  // ASSPAR4 + ACCELE (accele.F:63-123) + the acceleration part of BCS10 for node n
  auto node_acc = [&P](int n, R* a, R* ar) {
    a[0] = a[1] = a[2] = ar[0] = ar[1] = ar[2] = R(0);
    for (long k = P.adsky[n]; k < P.adsky[n + 1]; ++k) {
      const R* f = &P.fsky[8 * k];
      a[0] = a[0] + f[0]; a[1] = a[1] + f[1]; a[2] = a[2] + f[2];
      ar[0] = ar[0] + f[3]; ar[1] = ar[1] + f[4]; ar[2] = ar[2] + f[5];
    }
    R msn = P.ms[n];
    if (msn > R(0)) { R r = R(1) / msn; a[0] *= r; a[1] *= r; a[2] *= r; }
    else { a[0] = a[1] = a[2] = 0; }
    R inn = P.in[n];
    if (inn > R(0)) { R r = R(1) / inn; ar[0] *= r; ar[1] *= r; ar[2] *= r; }
    else { ar[0] = ar[1] = ar[2] = 0; }
  };
  auto skew_of = [&](int n) -> const double* { return P.iskew[n] >= 0 ? m.skews[P.iskew[n]].data() : nullptr; };
  auto bcs_acc = [&](int n, R* a, R* ar) {
    bcs1v(P.icodt[n], skew_of(n), a);
    bcs1v(P.icodr[n], skew_of(n), ar);
  };
  // RLINK10 / RLINK1 (resol.F:7053, rlink1.F): per link, MASS = sum MS, AX = sum MS*A
  // over its nodes after ACCELE and BCS10 (FRL6 sums in DOUBLE PRECISION), mean = AX/MASS
  const int N = P.numnod;
  std::vector<int> link_of;
  std::vector<std::array<double, 6>> link_mean;
  std::vector<std::array<int, 2>> link_dirs;
  for (auto& L : m.rlinks) {
    if (L.part != p || (L.ic == 0 && L.icr == 0)) continue;
    if (link_of.empty()) link_of.assign(N, -1);
    const int li = (int)link_mean.size();
    double S[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int n : L.nodes) {
      R a[3], ar[3];
      node_acc(n, a, ar);
      bcs_acc(n, a, ar);
      const R msn = P.ms[n], inn = P.in[n];
      S[0] += double(msn); S[1] += double(msn * a[0]); S[2] += double(msn * a[1]); S[3] += double(msn * a[2]);
      S[4] += double(inn); S[5] += double(inn * ar[0]); S[6] += double(inn * ar[1]); S[7] += double(inn * ar[2]);
      link_of[n] = li;
    }
    int ic = L.ic, icr = L.icr;
    if (S[0] == 0.0) ic = 0;          // rlink1.F: IF(MASS==ZERO)GOTO 250
    if (S[4] == 0.0) icr = 0;         // IF(INER==ZERO)RETURN
    link_mean.push_back({ic ? S[1] / S[0] : 0.0, ic ? S[2] / S[0] : 0.0, ic ? S[3] / S[0] : 0.0,
                         icr ? S[5] / S[4] : 0.0, icr ? S[6] / S[4] : 0.0, icr ? S[7] / S[4] : 0.0});
    link_dirs.push_back({ic, icr});
  }
  // rigid bodies: their nodes are updated after the others (RBYFOR, RBYVIT below)
  std::vector<char> rb_node;
  for (auto& rb : m.rbodies) {
    if (rb.part != p) continue;
    if (rb_node.empty()) rb_node.assign(N, 0);
    rb_node[rb.master] = 1;
    for (int n : rb.slaves) rb_node[n] = 2;
  }
  // ASSPAR4 + ACCELE + BCS10 + RLINK10 + BCS10 + (energies) + VELOCITY + DEPLA, per node
  std::vector<double> ek(last ? N : 0), ekr(last ? N : 0);
  int nan_node = -1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int n = 0; n < N; ++n) {
    if (!rb_node.empty() && rb_node[n]) continue;
    R a[3], ar[3];
    node_acc(n, a, ar);
    const R msn = P.ms[n], inn = P.in[n];
    if (!std::isfinite(double(a[0]) + double(a[1]) + double(a[2]))) nan_node = n;
    R* v = &P.v[3 * n];
    R* vr = &P.vr[3 * n];
    // BCS10 / BCS1V (bcs1.F:52-100): bit 4 = x, 2 = y, 1 = z, global or skew axes
    bcs1v(P.icodt[n], skew_of(n), v);
    bcs1v(P.icodr[n], skew_of(n), vr);
    bcs_acc(n, a, ar);
    if (!link_of.empty() && link_of[n] >= 0) {
      const int li = link_of[n];
      const auto& mu = link_mean[li];
      const int ic = link_dirs[li][0], icr = link_dirs[li][1];
      if (ic & 4) a[0] = R(mu[0]);
      if (ic & 2) a[1] = R(mu[1]);
      if (ic & 1) a[2] = R(mu[2]);
      if (icr & 4) ar[0] = R(mu[3]);
      if (icr & 2) ar[1] = R(mu[4]);
      if (icr & 1) ar[2] = R(mu[5]);
      bcs_acc(n, a, ar);              // resol.F:7458 reimposes the BCS
    }
    if (last) {   // ECRIT (ecrit.F:262-268, 315-322): DT05 = DT1/2
      double dt05 = 0.5 * DT1;
      double vx = double(v[0]) + dt05 * double(a[0]), vy = double(v[1]) + dt05 * double(a[1]), vz = double(v[2]) + dt05 * double(a[2]);
      ek[n] = (vx * vx + vy * vy + vz * vz) * 0.5 * double(msn);
      double wx = double(vr[0]) + dt05 * double(ar[0]), wy = double(vr[1]) + dt05 * double(ar[1]), wz = double(vr[2]) + dt05 * double(ar[2]);
      ekr[n] = (wx * wx + wy * wy + wz * wz) * 0.5 * double(inn);
    }
    // VELOCITY (velocity.F:56-84)
    v[0] = v[0] + DT12 * a[0]; v[1] = v[1] + DT12 * a[1]; v[2] = v[2] + DT12 * a[2];
    vr[0] = vr[0] + DT12 * ar[0]; vr[1] = vr[1] + DT12 * ar[1]; vr[2] = vr[2] + DT12 * ar[2];
    // DEPLA (displacement.F:69-100)
    for (int c = 0; c < 3; ++c) {
      double vdt = t.dt2 * double(v[c]);
      P.d[3 * n + c] = P.d[3 * n + c] + vdt;
      P.x[3 * n + c] = P.x[3 * n + c] + vdt;
    }
  }
  // RBYFOR (resol.F:5452) before ACCELE, RBYVIT (resol.F:7515) after BCS10, then
  // VELOCITY and DEPLA of the bodies' nodes; kinetic energy with the RBYCOR
  // correction (rgbcor.F: the secondary nodes' energy is the body's, whose
  // rotational part is taken in the principal frame)
  double ek_rb = 0, ekr_rb = 0;
  for (auto& rb : m.rbodies) {
    if (rb.part != p) continue;
    auto raw = [&P](int n, R* f, R* mo) {
      f[0] = f[1] = f[2] = mo[0] = mo[1] = mo[2] = R(0);
      for (long k = P.adsky[n]; k < P.adsky[n + 1]; ++k) {
        const R* g = &P.fsky[8 * k];
        f[0] = f[0] + g[0]; f[1] = f[1] + g[1]; f[2] = f[2] + g[2];
        mo[0] = mo[0] + g[3]; mo[1] = mo[1] + g[4]; mo[2] = mo[2] + g[5];
      }
    };
    const int M = rb.master;
    R af[3], am[3];
    raw(M, af, am);
    rgbodfp(rb, P, af, am, R(DT1), raw);
    // ACCELE and BCS10 of the main node
    R a[3], ar[3];
    const R msm = P.ms[M], inm = P.in[M];
    for (int c = 0; c < 3; ++c) {
      a[c] = msm > R(0) ? af[c] * (R(1) / msm) : R(0);
      ar[c] = inm > R(0) ? am[c] * (R(1) / inm) : R(0);
    }
    if (!std::isfinite(double(a[0]) + double(a[1]) + double(a[2]))) nan_node = M;
    R* vm = &P.v[3 * M];
    R* vrm = &P.vr[3 * M];
    bcs1v(P.icodt[M], skew_of(M), vm);
    bcs1v(P.icodr[M], skew_of(M), vrm);
    bcs_acc(M, a, ar);
    // RGBODV (rgbodv.F:91-119, more than two secondary nodes)
    const R dt2 = R(t.dt2);
    const R vg[3] = {vrm[0] + ar[0] * DT12, vrm[1] + ar[1] * DT12, vrm[2] + ar[2] * DT12};
    const R usdt = R(1) / DT12;
    std::vector<R> as(3 * rb.slaves.size()), ars(3 * rb.slaves.size());
    for (size_t i = 0; i < rb.slaves.size(); ++i) {
      const int n = rb.slaves[i];
      R* vn = &P.v[3 * n];
      R* vrn = &P.vr[3 * n];
      bcs1v(P.icodt[n], skew_of(n), vn);
      bcs1v(P.icodr[n], skew_of(n), vrn);
      ars[3 * i] = (vg[0] - vrn[0]) * usdt;
      ars[3 * i + 1] = (vg[1] - vrn[1]) * usdt;
      ars[3 * i + 2] = (vg[2] - vrn[2]) * usdt;
      const R dx = R(P.x[3 * n] - P.x[3 * M]), dy = R(P.x[3 * n + 1] - P.x[3 * M + 1]),
              dz = R(P.x[3 * n + 2] - P.x[3 * M + 2]);
      const R v1x2 = vg[0] * dy, v2x1 = vg[1] * dx, v2x3 = vg[1] * dz, v3x2 = vg[2] * dy, v3x1 = vg[2] * dx,
              v1x3 = vg[0] * dz;
      const R vx1 = v2x3 - v3x2, vx2 = v3x1 - v1x3, vx3 = v1x2 - v2x1;
      as[3 * i] = a[0] + (vm[0] + vx1 + R(0.5) * dt2 * (vg[1] * vx3 - vg[2] * vx2) - vn[0]) * usdt;
      as[3 * i + 1] = a[1] + (vm[1] + vx2 + R(0.5) * dt2 * (vg[2] * vx1 - vg[0] * vx3) - vn[1]) * usdt;
      as[3 * i + 2] = a[2] + (vm[2] + vx3 + R(0.5) * dt2 * (vg[0] * vx2 - vg[1] * vx1) - vn[2]) * usdt;
    }
    if (last) {   // ECRIT + RBYCOR: the body's mass on its main node, its rotation in the principal frame
      const double dt05 = 0.5 * DT1;
      const double vx = double(vm[0]) + dt05 * double(a[0]), vy = double(vm[1]) + dt05 * double(a[1]),
                   vz = double(vm[2]) + dt05 * double(a[2]);
      ek_rb += (vx * vx + vy * vy + vz * vz) * 0.5 * double(msm);
      const R h = R(dt05);
      const R w1 = vrm[0] + ar[0] * h, w2 = vrm[1] + ar[1] * h, w3 = vrm[2] + ar[2] * h;
      const R* rby = rb.rby;
      const R i1 = rby[0] * w1 + rby[1] * w2 + rby[2] * w3;
      const R i2 = rby[3] * w1 + rby[4] * w2 + rby[5] * w3;
      const R i3 = rby[6] * w1 + rby[7] * w2 + rby[8] * w3;
      ekr_rb += 0.5 * (double(rby[9]) * double(i1) * double(i1) + double(rby[10]) * double(i2) * double(i2) +
                       double(rby[11]) * double(i3) * double(i3));
    }
    // VELOCITY and DEPLA of the main and secondary nodes
    auto advance = [&](int n, const R* an, const R* arn) {
      R* v = &P.v[3 * n];
      R* vr = &P.vr[3 * n];
      v[0] = v[0] + DT12 * an[0]; v[1] = v[1] + DT12 * an[1]; v[2] = v[2] + DT12 * an[2];
      vr[0] = vr[0] + DT12 * arn[0]; vr[1] = vr[1] + DT12 * arn[1]; vr[2] = vr[2] + DT12 * arn[2];
      for (int c = 0; c < 3; ++c) {
        double vdt = t.dt2 * double(v[c]);
        P.d[3 * n + c] = P.d[3 * n + c] + vdt;
        P.x[3 * n + c] = P.x[3 * n + c] + vdt;
      }
    };
    for (size_t i = 0; i < rb.slaves.size(); ++i) advance(rb.slaves[i], &as[3 * i], &ars[3 * i]);
    advance(M, a, ar);
  }
  if (nan_node >= 0) { m.errcode = OR_E_NAN; m.errindex = nan_node; return OR_E_NAN; }
  if (last) {
    double s = 0, sr = 0;
    for (int n = 0; n < N; ++n) { s += ek[n]; sr += ekr[n]; }
    P.ekin = s + ek_rb; P.ekinr = sr + ekr_rb;
  }
  // TT=TT+DT2 (resol.F:8261)
  t.tt += t.dt2;
  t.ncycle += 1;
  return OR_OK;
}

struct Handle {
  int precision;
  Model<double> md;
  Model<float> mf;
  template <class F> auto with(F f) { return precision == OR_PREC_SPLIT ? f(mf) : f(md); }
};

template <class R>
int add_part(Model<R>& m, int numnod, const double* x, const double* v, const double* vr,
             const double* ms, const double* in, const int* icodt, const int* icodr) {
  PartData<R> P;
  P.numnod = numnod;
  P.x.assign(x, x + 3 * numnod);
  P.d.assign(3 * numnod, 0.0);
  P.v.resize(3 * numnod); P.vr.assign(3 * numnod, R(0));
  for (int i = 0; i < 3 * numnod; ++i) { P.v[i] = R(v[i]); if (vr) P.vr[i] = R(vr[i]); }
  P.ms.resize(numnod); P.in.assign(numnod, R(0));
  for (int i = 0; i < numnod; ++i) { P.ms[i] = R(ms[i]); if (in) P.in[i] = R(in[i]); }
  P.icodt.assign(icodt, icodt + numnod);
  P.icodr.assign(numnod, 0);
  if (icodr) P.icodr.assign(icodr, icodr + numnod);
  m.parts.push_back(std::move(P));
  return OR_OK;
}

// hexa volume with the SDERI3 formula (starter: the same Jacobian)
double hex_volume(const double* x, const int* n) {
  auto X = [&](int k, int c) { return x[3 * n[k] + c]; };
  double X17 = X(6,0)-X(0,0), X28 = X(7,0)-X(1,0), X35 = X(4,0)-X(2,0), X46 = X(5,0)-X(3,0);
  double Y17 = X(6,1)-X(0,1), Y28 = X(7,1)-X(1,1), Y35 = X(4,1)-X(2,1), Y46 = X(5,1)-X(3,1);
  double Z17 = X(6,2)-X(0,2), Z28 = X(7,2)-X(1,2), Z35 = X(4,2)-X(2,2), Z46 = X(5,2)-X(3,2);
  double J1 = X17+X28-X35-X46, J2 = Y17+Y28-Y35-Y46, J3 = Z17+Z28-Z35-Z46;
  double J4 = X17+X46+X28+X35, J5 = Y17+Y46+Y28+Y35, J6 = Z17+Z46+Z28+Z35;
  double J7 = X17+X46-X28-X35, J8 = Y17+Y46-Y28-Y35, J9 = Z17+Z46-Z28-Z35;
  return (1.0/64.0)*(J1*(J5*J9-J6*J8) + J2*(J6*J7-J4*J9) + J3*(J4*J8-J5*J7));
}

template <class R>
int add_hex(Model<R>& m, int part, int nel, const int* ixs, const or_material* mat,
            const or_solid_prop* prop, const double* vol0) {
  HexGroup<R> g;
  g.part = part; g.nel = nel; g.mat = *mat; g.prop = *prop;
  g.gofs = m.parts[part].nel_solid;
  m.parts[part].nel_solid += nel;
  g.ix.resize(8 * nel);
  for (int e = 0; e < nel; ++e) for (int k = 0; k < 8; ++k) g.ix[8 * e + k] = ixs[11 * e + 1 + k] - 1;
  g.sig.assign(6 * nel, R(0));
  g.eint.assign(nel, R(0)); g.qvis.assign(nel, R(0)); g.off.assign(nel, R(1));
  g.pla.assign(nel, R(0)); g.epsd.assign(nel, R(0));
  g.rho.assign(nel, R(mat->rho0));
  g.vol0.resize(nel); g.vol0dp.resize(nel);
  for (int e = 0; e < nel; ++e) {
    double v = vol0 ? vol0[e] : hex_volume(m.parts[part].x.data(), &g.ix[8 * e]);
    g.vol0[e] = R(v); g.vol0dp[e] = v;
  }
  m.hex.push_back(std::move(g));
  return OR_OK;
}

template <class R>
int add_shell(Model<R>& m, int part, int nel, const int* ixc, const or_material* mat,
              const or_shell_prop* prop, const double* thke) {
  if (prop->npt < 1 || prop->npt > 10 || prop->ipla < 0 || prop->ipla > 2) return OR_E_UNSUPPORTED;
  if (prop->ishell < 0 || prop->ishell > 4 || !(prop->dn >= 0)) return OR_E_UNSUPPORTED;
  if (prop->ishfram != 0 && prop->ishfram != 2) return OR_E_UNSUPPORTED;
  ShellGroup<R> g;
  g.part = part; g.nel = nel; g.mat = *mat; g.prop = *prop;
  g.gofs = m.parts[part].nel_shell;
  m.parts[part].nel_shell += nel;
  g.ix.resize(4 * nel);
  for (int e = 0; e < nel; ++e) for (int k = 0; k < 4; ++k) g.ix[4 * e + k] = ixc[7 * e + 1 + k] - 1;
  g.thke.resize(nel); g.thk.resize(nel);
  for (int e = 0; e < nel; ++e) { g.thke[e] = R(thke ? thke[e] : prop->thk); g.thk[e] = g.thke[e]; }
  g.hourg.assign(3 * nel, R(0)); g.eint.assign(2 * nel, R(0));
  g.sig.assign(prop->npt * 5 * nel, R(0)); g.pla.assign(prop->npt * nel, R(0));
  m.shell.push_back(std::move(g));
  return OR_OK;
}

} // namespace

extern "C" {

void* oracle_create(const or_ecycle_config* cfg) {
  Handle* h = new Handle();
  h->precision = cfg->precision;
  h->md.cfg = *cfg; h->mf.cfg = *cfg;
  return h;
}
void oracle_destroy(void* hh) { delete (Handle*)hh; }

int oracle_add_part(void* hh, int numnod, const double* x, const double* v, const double* vr,
                    const double* ms, const double* in, const int* icodt, const int* icodr) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) { return add_part(m, numnod, x, v, vr, ms, in, icodt, icodr); });
}
int oracle_add_hex_group(void* hh, int part, int nel, const int* ixs, const or_material* mat,
                         const or_solid_prop* prop, const double* vol0) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) { return add_hex(m, part, nel, ixs, mat, prop, vol0); });
}
int oracle_add_shell_group(void* hh, int part, int nel, const int* ixc, const or_material* mat,
                           const or_shell_prop* prop, const double* thke) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) { return add_shell(m, part, nel, ixc, mat, prop, thke); });
}
int oracle_set_shell_yield(void* hh, int gi, const double* jc_a) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    auto& g = m.shell[gi];
    g.jca.resize(g.nel);
    for (int i = 0; i < g.nel; ++i) g.jca[i] = jc_a[i];
    return (int)OR_OK;
  });
}
int oracle_add_rlink(void* hh, int part, int nnod, const int* nodes, int ic, int icr) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    if (part < 0 || part >= (int)m.parts.size() || nnod < 1 || !nodes || ic < 0 || ic > 7 || icr < 0 || icr > 7)
      return (int)OR_E_ARG;
    RLink L;
    L.part = part; L.ic = ic; L.icr = icr;
    for (int i = 0; i < nnod; ++i) {
      if (nodes[i] < 1 || nodes[i] > m.parts[part].numnod) return (int)OR_E_ARG;
      L.nodes.push_back(nodes[i] - 1);
    }
    m.rlinks.push_back(std::move(L));
    return (int)OR_OK;
  });
}
// A rigid body after the starter's initialisation: main node and nsl secondary
// nodes (1-based), rby12 = principal axes e1, e2, e3 and principal inertias; the
// main node's mass, inertia and position are those of add_part (the body's).
int oracle_add_rbody(void* hh, int part, int master, int nsl, const int* slaves, const double* rby12) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    typedef typename std::remove_reference<decltype(m)>::type::real_t R;
    if (part < 0 || part >= (int)m.parts.size() || nsl < 3 || !slaves || !rby12) return (int)OR_E_ARG;
    const int nn = m.parts[part].numnod;
    if (master < 1 || master > nn) return (int)OR_E_ARG;
    RBody<R> rb;
    rb.part = part; rb.master = master - 1;
    for (int i = 0; i < nsl; ++i) {
      if (slaves[i] < 1 || slaves[i] > nn || slaves[i] == master) return (int)OR_E_ARG;
      rb.slaves.push_back(slaves[i] - 1);
    }
    for (int k = 0; k < 12; ++k) rb.rby[k] = R(rby12[k]);
    m.rbodies.push_back(std::move(rb));
    return (int)OR_OK;
  });
}
int oracle_set_rlink(void* hh, int link, int ic, int icr) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    if (link < 0 || link >= (int)m.rlinks.size() || ic < 0 || ic > 7 || icr < 0 || icr > 7) return (int)OR_E_ARG;
    m.rlinks[link].ic = ic; m.rlinks[link].icr = icr;
    return (int)OR_OK;
  });
}
int oracle_add_function(void* hh, int npts, const double* x, const double* y) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    if (npts < 1 || !x || !y) return (int)OR_E_ARG;
    Func f;
    f.x.assign(x, x + npts); f.y.assign(y, y + npts);
    m.funcs.push_back(std::move(f));
    return (int)OR_OK;
  });
}
int oracle_add_cload(void* hh, int part, int nnod, const int* nodes, int dir, int skew, int func,
                     double ascale_x, double fscale) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    if (part < 0 || part >= (int)m.parts.size() || dir < 1 || dir > 6 || func < 0 || func >= (int)m.funcs.size() ||
        skew < -1 || skew >= (int)m.skews.size() || ascale_x == 0.0)
      return (int)OR_E_ARG;
    for (int i = 0; i < nnod; ++i) {
      if (nodes[i] < 1 || nodes[i] > m.parts[part].numnod) return (int)OR_E_ARG;
      m.cloads.push_back(CLoad{part, nodes[i] - 1, dir, skew, func, 1.0 / ascale_x, fscale, -1});
    }
    return (int)OR_OK;
  });
}
int oracle_add_pload(void* hh, int part, int nseg, const int* seg, int func, double ascale_x, double fscale) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    if (part < 0 || part >= (int)m.parts.size() || func < 0 || func >= (int)m.funcs.size() || ascale_x == 0.0)
      return (int)OR_E_ARG;
    for (int i = 0; i < nseg; ++i) {
      PLoad q{};
      q.part = part; q.func = func; q.fcx = 1.0 / ascale_x; q.fcy = fscale;
      for (int k = 0; k < 4; ++k) q.n[k] = seg[4 * i + k] - 1;     // n4 = 0 -> -1: triangle
      for (int k = 0; k < 4; ++k)
        if ((k < 3 || q.n[3] >= 0) && (q.n[k] < 0 || q.n[k] >= m.parts[part].numnod)) return (int)OR_E_ARG;
      m.ploads.push_back(q);
    }
    return (int)OR_OK;
  });
}
int oracle_add_skew(void* hh, const double* axes9) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    std::array<double, 9> a;
    for (int k = 0; k < 9; ++k) a[k] = axes9[k];
    m.skews.push_back(a);
    return (int)OR_OK;
  });
}
int oracle_set_bcs_skew(void* hh, int part, const int* skew) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    if (part < 0 || part >= (int)m.parts.size()) return (int)OR_E_ARG;
    auto& P = m.parts[part];
    P.iskew.assign(skew, skew + P.numnod);
    for (int s : P.iskew) if (s < -1 || s >= (int)m.skews.size()) return (int)OR_E_ARG;
    return (int)OR_OK;
  });
}
int oracle_finalize(void* hh) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) { build_skyline(m); m.finalized = true; return OR_OK; });
}
int oracle_step(void* hh, int ncycles, or_ecycle_time* t, int nthreads) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    for (int c = 0; c < ncycles; ++c)
      for (size_t p = 0; p < m.parts.size(); ++p) {
        int s = cycle(m, (int)p, t[p], nthreads, c == ncycles - 1);
        if (s) return s;
      }
    return (int)OR_OK;
  });
}
int oracle_get_nodes(void* hh, int part, double* x, double* d, double* v, double* vr) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    auto& P = m.parts[part];
    for (int i = 0; i < 3 * P.numnod; ++i) {
      if (x) x[i] = P.x[i];
      if (d) d[i] = P.d[i];
      if (v) v[i] = P.v[i];
      if (vr) vr[i] = P.vr[i];
    }
    return (int)OR_OK;
  });
}
int oracle_get_hex_state(void* hh, int gi, double* sig, double* eint, double* rho, double* qvis,
                         double* pla, double* epsd) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    auto& g = m.hex[gi];
    for (int i = 0; i < 6 * g.nel; ++i) if (sig) sig[i] = g.sig[i];
    for (int i = 0; i < g.nel; ++i) {
      if (eint) eint[i] = g.eint[i];
      if (rho) rho[i] = g.rho[i];
      if (qvis) qvis[i] = g.qvis[i];
      if (pla) pla[i] = g.pla[i];
      if (epsd) epsd[i] = g.epsd[i];
    }
    return (int)OR_OK;
  });
}
int oracle_get_shell_state(void* hh, int gi, double* sig, double* pla, double* thk, double* hourg,
                           double* eint) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    auto& g = m.shell[gi];
    for (size_t i = 0; i < g.sig.size(); ++i) if (sig) sig[i] = g.sig[i];
    for (size_t i = 0; i < g.pla.size(); ++i) if (pla) pla[i] = g.pla[i];
    for (int i = 0; i < g.nel; ++i) if (thk) thk[i] = g.thk[i];
    for (int i = 0; i < 3 * g.nel; ++i) if (hourg) hourg[i] = g.hourg[i];
    for (int i = 0; i < 2 * g.nel; ++i) if (eint) eint[i] = g.eint[i];
    return (int)OR_OK;
  });
}
int oracle_energies(void* hh, int part, or_energies* e) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) {
    auto& P = m.parts[part];
    double ei = 0;
    for (auto& g : m.hex) if (g.part == part) for (int i = 0; i < g.nel; ++i) ei += double(g.eint[i]) * double(g.vol0[i]);
    for (auto& g : m.shell) if (g.part == part) for (int i = 0; i < g.nel; ++i) ei += double(g.eint[i]) + double(g.eint[g.nel + i]);
    e->internal = ei; e->kinetic = P.ekin; e->kinetic_rot = P.ekinr;
    e->hourglass = P.ehour; e->plastic_work = P.wplast; e->external_work = P.wext;
    return (int)OR_OK;
  });
}
int oracle_error_info(void* hh, int* code, int* index) {
  Handle* h = (Handle*)hh;
  return h->with([&](auto& m) { *code = m.errcode; *index = m.errindex; return (int)OR_OK; });
}

} // extern "C"
