// ecycle_noalloc.cu -- an element-cycle entry point that allocates nothing.
//
// Some callers cannot let a library allocate device memory: an engine that
// places every array in a device pool it reserves at start-up, so that its
// footprint stays fixed and known during the whole time loop, has no room for
// a library's own cudaMalloc calls.  or_ecycle_hex_step_noalloc serves them:
// the caller passes every input and output as device pointers it owns, and the
// only intermediate buffer, the Parith/ON force skyline FSKY (one slot per
// element corner, asspar4.F:160-175), lives in a file-scope static device array
// of fixed size.  The function calls no cudaMalloc, cudaFree or other
// allocating routine, on the host or on the device.
//
// Limits and sharing rules:
//   * at most OR_NOALLOC_MAX_SLOTS skyline slots (8 per hexa, i.e. 32,768
//     hexas); larger groups are rejected with OR_E_ARG;
//   * FP64 only, one hexa group of one part, LAW1 or LAW2;
//   * every GPU that loads the library holds the scratch (8 MB) until exit;
//   * the caller's tables are checked on the device before the first cycle:
//     every connectivity entry in [0, numnod), ADSKY a CSR over 8*nel slots
//     (ADSKY(1) = 0, ascending, ADSKY(numnod+1) = 8*nel) and IADS a permutation
//     of [0, 8*nel) that puts each corner among its own node's slots; a table
//     that fails is rejected with OR_E_ARG before anything is written, and the
//     kernels also skip any slot outside the scratch;
//   * every call shares the scratch and it keeps the last call's contents:
//     the time-step accumulator, error word and slot counters are cleared at
//     the start of each call, the skyline slots are all rewritten every cycle;
//     calls that overlap on the GPU (other streams, other host threads) race
//     on it;
//   * the first call on a device looks the scratch's device address up once
//     (cudaGetSymbolAddress, under a lock) with that device current;
//   * the call is synchronous: it waits for its own work with the bounded
//     event poll of the handle path (OR_ECYCLE_TIMEOUT_S, default 900 s), so
//     it cannot be recorded into a CUDA graph by stream capture.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <thread>
#include <cuda_runtime.h>

#include "../../include/or_ecycle.h"

namespace {

constexpr int NOALLOC_TILE = 128;

struct NoallocScalars {
  unsigned long long dtbits;   // min over elements of the element dt (double bits)
  unsigned long long dtkey;    // min of (float(dt) bits << 32 | 0x80000000 | element): NELTS
  int err_code;
  int err_index;
  double time[8];              // tt, dt1, dt2, dt12, dt2old, ncycle, ityptst, neltst
};

// the shared scratch: FSKY slots (fx, fy, fz, unused) and the per-call scalars
static __device__ __align__(256) double4 g_fsky_scratch[OR_NOALLOC_MAX_SLOTS];
static __device__ __align__(256) NoallocScalars g_noalloc_scalars;

struct ScratchPtrs {
  double4* fsky;
  NoallocScalars* sc;
};

constexpr int MAX_DEVICES = 64;
ScratchPtrs g_ptrs[MAX_DEVICES];
bool g_ptrs_ready[MAX_DEVICES];
std::mutex g_ptrs_lock;          // first calls from several host threads

__device__ inline void noalloc_error(NoallocScalars* sc, int code, int index) {
  if (atomicCAS(&sc->err_code, 0, code) == 0) sc->err_index = index;
}

// Table check, one thread per element corner (the scratch's first 8*nel words
// count the corners that land on each slot): the corner's node is in
// [0, numnod), its slot is in [0, 8*nel) and among its node's ADSKY range, and
// no other corner took the slot.  With ADSKY checked by check_adsky_kernel this
// makes IADS a permutation that fills every node's range exactly.
__global__ void check_corners_kernel(int nel, int numnod, const int* __restrict__ conn, const int* __restrict__ iads,
                                     const int* __restrict__ adsky, unsigned* count, NoallocScalars* sc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= 8 * nel) return;
  const int e = c >> 3, n = conn[c], s = iads[c], nslot = 8 * nel;
  if (n < 0 || n >= numnod || s < 0 || s >= nslot) { noalloc_error(sc, OR_E_ARG, e); return; }
  if (s < adsky[n] || s >= adsky[n + 1]) { noalloc_error(sc, OR_E_ARG, e); return; }
  if (atomicAdd(&count[s], 1u) != 0u) noalloc_error(sc, OR_E_ARG, e);
}

// ADSKY check, one thread per node: ADSKY(1) = 0, ascending, ADSKY(numnod+1) = 8*nel
__global__ void check_adsky_kernel(int nel, int numnod, const int* __restrict__ adsky, NoallocScalars* sc) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= numnod) return;
  const int a0 = adsky[n], a1 = adsky[n + 1];
  if (a1 < a0 || (n == 0 && a0 != 0) || (n == numnod - 1 && a1 != 8 * nel)) noalloc_error(sc, OR_E_ARG, n);
}

// One thread per hexa: SDERI3, SDLEN3, SDEFO3, SRHO3, SROTA3, M1LAW / M2LAW with
// MQVISCB, SHVIS3, SFINT3, then SCUMU3P writes of the 8 corner forces into the
// skyline slots IADS(k, e) given by the caller (FP64 throughout).
__global__ void __launch_bounds__(NOALLOC_TILE)
hex_fsky_kernel(int nel, const int* __restrict__ conn, const int* __restrict__ iads,
                const double* __restrict__ x, const double* __restrict__ v,
                double* sig, double* eint, double* rho, double* qvis, double* pla, double* epsd,
                const double* __restrict__ vol0, or_material mt, or_solid_prop pr, double dtfac,
                double4* fsky, NoallocScalars* sc) {
  const int e = blockIdx.x * NOALLOC_TILE + threadIdx.x;
  __shared__ unsigned long long s_min[NOALLOC_TILE / 32], s_key[NOALLOC_TILE / 32];
  unsigned long long mybits = ~0ull, mykey = ~0ull;
  if (e < nel) {
    const double DT1 = sc->time[1];
    double XD[8], YD[8], ZD[8], VX[8], VY[8], VZ[8];
    int nd[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      nd[k] = conn[8 * e + k];
      XD[k] = x[3 * nd[k]]; YD[k] = x[3 * nd[k] + 1]; ZD[k] = x[3 * nd[k] + 2];
      VX[k] = v[3 * nd[k]]; VY[k] = v[3 * nd[k] + 1]; VZ[k] = v[3 * nd[k] + 2];
    }
    // SDERI3 (sderi3.F:103-149, 264-298)
    const double X17 = XD[6] - XD[0], X28 = XD[7] - XD[1], X35 = XD[4] - XD[2], X46 = XD[5] - XD[3];
    const double Y17 = YD[6] - YD[0], Y28 = YD[7] - YD[1], Y35 = YD[4] - YD[2], Y46 = YD[5] - YD[3];
    const double Z17 = ZD[6] - ZD[0], Z28 = ZD[7] - ZD[1], Z35 = ZD[4] - ZD[2], Z46 = ZD[5] - ZD[3];
    const double J1 = X17 + X28 - X35 - X46, J2 = Y17 + Y28 - Y35 - Y46, J3 = Z17 + Z28 - Z35 - Z46;
    const double xa = X17 + X46, xb = X28 + X35, ya = Y17 + Y46, yb = Y28 + Y35, za = Z17 + Z46, zb = Z28 + Z35;
    const double J4 = xa + xb, J5 = ya + yb, J6 = za + zb, J7 = xa - xb, J8 = ya - yb, J9 = za - zb;
    const double C1 = J5 * J9 - J6 * J8, C4 = J6 * J7 - J4 * J9, C7 = J4 * J8 - J5 * J7;
    double VOLN = (1.0 / 64.0) * (J1 * C1 + J2 * C4 + J3 * C7);
    if (!(VOLN > 0.0)) { noalloc_error(sc, OR_E_NEGVOL, e); VOLN = 1.0; }
    const double dett = (1.0 / 64.0) / VOLN;
    const double I1 = dett * C1, I4 = dett * C4, I7 = dett * C7;
    const double I2 = dett * (J3 * J8 - J2 * J9), I5 = dett * (J1 * J9 - J3 * J7), I8 = dett * (J2 * J7 - J1 * J8);
    const double I3 = dett * (J2 * J6 - J3 * J5), I6 = dett * (J3 * J4 - J1 * J6), I9 = dett * (J1 * J5 - J2 * J4);
    double PX[4], PY[4], PZ[4];
    {
      const double a12 = I1 + I2, a45 = I4 + I5, a78 = I7 + I8, b12 = I1 - I2, b45 = I4 - I5, b78 = I7 - I8;
      PX[0] = -a12 - I3; PY[0] = -a45 - I6; PZ[0] = -a78 - I9;
      PX[1] = -a12 + I3; PY[1] = -a45 + I6; PZ[1] = -a78 + I9;
      PX[2] = b12 + I3;  PY[2] = b45 + I6;  PZ[2] = b78 + I9;
      PX[3] = b12 - I3;  PY[3] = b45 - I6;  PZ[3] = b78 - I9;
    }
    const int HM[3][8] = {{1, -1, 1, -1, 1, -1, 1, -1}, {1, 1, -1, -1, -1, -1, 1, 1}, {1, -1, -1, 1, -1, 1, 1, -1}};
    double PXH[4][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double hx = 0, hy = 0, hz = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) { hx += HM[j][k] * XD[k]; hy += HM[j][k] * YD[k]; hz += HM[j][k] * ZD[k]; }
#pragma unroll
      for (int q = 0; q < 4; ++q) PXH[q][j] = PX[q] * hx + PY[q] * hy + PZ[q] * hz;
    }
    // SDLEN3 / SLEN (sdlen3.F:110-166)
    double AREAM = 1e-20;
    {
      const int FC[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const double x13 = XD[FC[f][2]] - XD[FC[f][0]], x24 = XD[FC[f][3]] - XD[FC[f][1]];
        const double y13 = YD[FC[f][2]] - YD[FC[f][0]], y24 = YD[FC[f][3]] - YD[FC[f][1]];
        const double z13 = ZD[FC[f][2]] - ZD[FC[f][0]], z24 = ZD[FC[f][3]] - ZD[FC[f][1]];
        const double s1 = x13 - x24, t1 = x13 + x24, s2 = y13 - y24, t2 = y13 + y24, s3 = z13 - z24, t3 = z13 + z24;
        const double E = s1 * s1 + s2 * s2 + s3 * s3, Fm = s1 * t1 + s2 * t2 + s3 * t3, G = t1 * t1 + t2 * t2 + t3 * t3;
        AREAM = fmax(E * G - Fm * Fm, AREAM);
      }
    }
    const double DELTAX = 4.0 * VOLN / sqrt(AREAM);
    // SDEFO3 (sdefo3.F:114-170)
    const double vx17 = VX[0] - VX[6], vx28 = VX[1] - VX[7], vx35 = VX[2] - VX[4], vx46 = VX[3] - VX[5];
    const double vy17 = VY[0] - VY[6], vy28 = VY[1] - VY[7], vy35 = VY[2] - VY[4], vy46 = VY[3] - VY[5];
    const double vz17 = VZ[0] - VZ[6], vz28 = VZ[1] - VZ[7], vz35 = VZ[2] - VZ[4], vz46 = VZ[3] - VZ[5];
    const double DXX = PX[0] * vx17 + PX[1] * vx28 + PX[2] * vx35 + PX[3] * vx46;
    const double DYY = PY[0] * vy17 + PY[1] * vy28 + PY[2] * vy35 + PY[3] * vy46;
    const double DZZ = PZ[0] * vz17 + PZ[1] * vz28 + PZ[2] * vz35 + PZ[3] * vz46;
    const double DXY = PY[0] * vx17 + PY[1] * vx28 + PY[2] * vx35 + PY[3] * vx46;
    const double DXZ = PZ[0] * vx17 + PZ[1] * vx28 + PZ[2] * vx35 + PZ[3] * vx46;
    const double DYX = PX[0] * vy17 + PX[1] * vy28 + PX[2] * vy35 + PX[3] * vy46;
    const double DYZ = PZ[0] * vy17 + PZ[1] * vy28 + PZ[2] * vy35 + PZ[3] * vy46;
    const double DZX = PX[0] * vz17 + PX[1] * vz28 + PX[2] * vz35 + PX[3] * vz46;
    const double DZY = PY[0] * vz17 + PY[1] * vz28 + PY[2] * vz35 + PY[3] * vz46;
    const double D4 = DXY + DYX, D5 = DYZ + DZY, D6 = DXZ + DZX;
    const double WZZ = 0.5 * DT1 * (DYX - DXY), WYY = 0.5 * DT1 * (DXZ - DZX), WXX = 0.5 * DT1 * (DZY - DYZ);
    // SRHO3 (srho3.F:122-156)
    const double RHO0 = mt.rho0, VOLO = vol0[e];
    const double DVOL = VOLN - (RHO0 / rho[e]) * VOLO;
    const double RHON = RHO0 * (VOLO / VOLN);
    const double AMU = RHON / RHO0 - 1.0;
    double EINT = eint[e] * VOLO;
    // SROTA3 (srota3.F:81-91)
    const double S1 = sig[0 * nel + e], S2 = sig[1 * nel + e], S3 = sig[2 * nel + e];
    const double S4 = sig[3 * nel + e], S5 = sig[4 * nel + e], S6 = sig[5 * nel + e];
    double SG[6];
    {
      const double q1 = 2.0 * S4 * WZZ, q2 = 2.0 * S6 * WYY, q3 = 2.0 * S5 * WXX;
      SG[0] = S1 - q1 + q2; SG[1] = S2 + q1 - q3; SG[2] = S3 - q2 + q3;
      SG[3] = S4 + WZZ * (S1 - S2) + WYY * S5 - WXX * S6;
      SG[4] = S5 + WXX * (S2 - S3) + WZZ * S6 - WYY * S4;
      SG[5] = S6 + WYY * (S3 - S1) + WXX * S4 - WZZ * S5;
    }
    // elastic predictor (m1law.F:124-140, m2law.F:187-200)
    const double G = mt.shear, G1 = DT1 * G, G2 = 2.0 * G1;
    const double SSP = sqrt((1.333 * G + mt.bulk) / RHO0);
    {
      const double P = -(1.0 / 3.0) * (SG[0] + SG[1] + SG[2]);
      const double DAV = -(1.0 / 3.0) * (DXX + DYY + DZZ);
      SG[0] += P + G2 * (DXX + DAV); SG[1] += P + G2 * (DYY + DAV); SG[2] += P + G2 * (DZZ + DAV);
      SG[3] += G1 * D4; SG[4] += G1 * D5; SG[5] += G1 * D6;
    }
    if (mt.law == OR_LAW_JOHNSON_COOK) {
      // radial return (m2law.F:197-352), CC = 0, FISOKIN = 0
      double AJ2 = 0.5 * (SG[0] * SG[0] + SG[1] * SG[1] + SG[2] * SG[2]) + SG[3] * SG[3] + SG[4] * SG[4] + SG[5] * SG[5];
      AJ2 = sqrt(3.0 * AJ2);
      const double e4 = 0.5 * D4, e5 = 0.5 * D5, e6 = 0.5 * D6;
      epsd[e] = sqrt(DXX * DXX + DYY * DYY + DZZ * DZZ + 2.0 * (e4 * e4 + e5 * e5 + e6 * e6));
      const double CA = mt.jc_a, CB = mt.jc_b, CN = mt.jc_n;
      const double EPXE = pla[e];
      double AK, QH;
      if (CN == 1.0) { AK = CA + CB * EPXE; QH = CB; }
      else if (EPXE > 0.0) {
        AK = CA + CB * pow(EPXE, CN);
        QH = CN > 1.0 ? CB * CN * pow(EPXE, CN - 1.0) : CB * CN / pow(EPXE, 1.0 - CN);
      } else { AK = CA; QH = 0.0; }
      if (mt.sigmax < AK) { AK = mt.sigmax; QH = 0.0; }
      if (EPXE > mt.epsmax) { AK = 0.0; QH = 0.0; }
      const double SCALE0 = fmin(1.0, AK / fmax(AJ2, 1e-15));
      const double DPLA = (1.0 - SCALE0) * AJ2 / fmax(3.0 * G + QH, 1e-15);
      AK = AK + DPLA * QH;
      const double SCALE = fmin(1.0, AK / fmax(AJ2, 1e-15));
#pragma unroll
      for (int c = 0; c < 6; ++c) SG[c] *= SCALE;
      pla[e] = EPXE + DPLA;
    }
    // MQVISCB (mqviscb.F:139-354)
    const double DD = -DXX - DYY - DZZ;
    const double AL = cbrt(VOLN), AD = fmax(0.0, DD);
    const double QAA = pr.qa * pr.qa * AD;
    const double QX = pr.qb * SSP + AL * QAA;
    const double QNEW = RHON * AD * AL * (QAA * AL + pr.qb * SSP);
    const double SSP_EQ = fmax(1e-20, QX + sqrt(QX * QX + SSP * SSP));
    const double DTX = dtfac * (DELTAX / SSP_EQ);
    mybits = (unsigned long long)__double_as_longlong(DTX);
    mykey = ((unsigned long long)__float_as_uint((float)DTX) << 32) | (0x80000000u | (unsigned)e);
    // pressure and internal energy (m1law.F:172-190, m2law.F:434-461)
    const double PNEW = mt.bulk * AMU;
    SG[0] -= PNEW; SG[1] -= PNEW; SG[2] -= PNEW;
    const double DTA = 0.5 * DT1;
    const double VOL_AVG = VOLN - 0.5 * DVOL;
    double EINC;
    if (mt.law == OR_LAW_ELASTIC) {
      const double P2 = -(S1 + SG[0] + S2 + SG[1] + S3 + SG[2]) * (1.0 / 3.0);
      EINC = VOL_AVG * (DXX * (S1 + SG[0] + P2) + DYY * (S2 + SG[1] + P2) + DZZ * (S3 + SG[2] + P2) +
                        D4 * (S4 + SG[3]) + D5 * (S5 + SG[4]) + D6 * (S6 + SG[5])) * DTA -
             0.5 * DVOL * (qvis[e] + QNEW + P2);
    } else {
      EINC = VOL_AVG * (DXX * (S1 + SG[0]) + DYY * (S2 + SG[1]) + DZZ * (S3 + SG[2]) +
                        D4 * (S4 + SG[3]) + D5 * (S5 + SG[4]) + D6 * (S6 + SG[5])) * DTA -
             0.5 * DVOL * (qvis[e] + QNEW);
    }
    EINT = (EINT + EINC) / fmax(1e-15, VOLO);
#pragma unroll
    for (int c = 0; c < 6; ++c) sig[c * nel + e] = SG[c];
    eint[e] = EINT; rho[e] = RHON; qvis[e] = QNEW;
    // SHVIS3 (shvis3.F:156-424), JHBE >= 1
    double F[3][8];
    {
      const double CAQ = 0.25 * pr.qh;
      double FCL = CAQ * RHON * (AL * AL);
      const double FCQ = FCL * CAQ * 100.0;
      FCL *= SSP;
      double Gv[3][8];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        Gv[j][0] = HM[j][0] - PXH[0][j]; Gv[j][1] = HM[j][1] - PXH[1][j];
        Gv[j][2] = HM[j][2] - PXH[2][j]; Gv[j][3] = HM[j][3] - PXH[3][j];
        Gv[j][4] = HM[j][4] + PXH[2][j]; Gv[j][5] = HM[j][5] + PXH[3][j];
        Gv[j][6] = HM[j][6] + PXH[0][j]; Gv[j][7] = HM[j][7] + PXH[1][j];
      }
      const int h4[8] = {1, -1, 1, -1, -1, 1, -1, 1};
      double HX[4], HY[4], HZ[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        double hx = 0, hy = 0, hz = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const double g = j < 3 ? Gv[j][k] : (double)h4[k];
          hx += g * VX[k]; hy += g * VY[k]; hz += g * VZ[k];
        }
        HX[j] = hx * (FCL + fabs(hx) * FCQ);
        HY[j] = hy * (FCL + fabs(hy) * FCQ);
        HZ[j] = hz * (FCL + fabs(hz) * FCQ);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        F[0][k] = -Gv[0][k] * HX[0] - Gv[1][k] * HX[1] - Gv[2][k] * HX[2] - h4[k] * HX[3];
        F[1][k] = -Gv[0][k] * HY[0] - Gv[1][k] * HY[1] - Gv[2][k] * HY[2] - h4[k] * HY[3];
        F[2][k] = -Gv[0][k] * HZ[0] - Gv[1][k] * HZ[1] - Gv[2][k] * HZ[2] - h4[k] * HZ[3];
      }
    }
    // SFINT3 (sfint3.F:256-321)
    {
      const double s1 = (SG[0] - QNEW) * VOLN, s2 = (SG[1] - QNEW) * VOLN, s3 = (SG[2] - QNEW) * VOLN;
      const double s4 = SG[3] * VOLN, s5 = SG[4] * VOLN, s6 = SG[5] * VOLN;
      const int n1[4] = {0, 1, 2, 3}, n2[4] = {6, 7, 4, 5};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double f = s1 * PX[q] + s4 * PY[q] + s6 * PZ[q];
        F[0][n1[q]] -= f; F[0][n2[q]] += f;
        f = s2 * PY[q] + s4 * PX[q] + s5 * PZ[q];
        F[1][n1[q]] -= f; F[1][n2[q]] += f;
        f = s3 * PZ[q] + s6 * PX[q] + s5 * PY[q];
        F[2][n1[q]] -= f; F[2][n2[q]] += f;
      }
    }
    // SCUMU3P (scumu3p.F:205-260): one skyline slot per corner; the tables were
    // checked before the first cycle, and a slot outside the scratch is skipped
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int s = iads[8 * e + k];
      if ((unsigned)s < (unsigned)(8 * nel)) fsky[s] = make_double4(F[0][k], F[1][k], F[2][k], 0.0);
      else noalloc_error(sc, OR_E_ARG, e);
    }
  }
  // element dt min-reduction (exact bits, and the key that names the element):
  // warp shuffles, then one atomicMin of each per block
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long b = __shfl_xor_sync(0xffffffffu, mybits, o);
    const unsigned long long k = __shfl_xor_sync(0xffffffffu, mykey, o);
    mybits = b < mybits ? b : mybits;
    mykey = k < mykey ? k : mykey;
  }
  if ((threadIdx.x & 31) == 0) { s_min[threadIdx.x >> 5] = mybits; s_key[threadIdx.x >> 5] = mykey; }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = s_min[0], q = s_key[0];
    for (int w = 1; w < NOALLOC_TILE / 32; ++w) {
      m = s_min[w] < m ? s_min[w] : m;
      q = s_key[w] < q ? s_key[w] : q;
    }
    atomicMin(&sc->dtbits, m);
    atomicMin(&sc->dtkey, q);
  }
}

// dt logic (resol.F:5853-6226) by one thread, then ASSPAR4 + ACCELE + BCS10 +
// VELOCITY + DEPLA per node.  The dt state is advanced by the last block to finish.
__global__ void dt_kernel(NoallocScalars* sc, double growth, double dtmx) {
  double* t = sc->time;   // tt, dt1, dt2, dt12, dt2old, ncycle
  const double dt2t = __longlong_as_double((long long)sc->dtbits);
  double DT2 = 1e6;
  if (sc->dtbits != ~0ull && dt2t < DT2) {   // the element that set DT2 (ITYPTS = 1, NELTS)
    DT2 = dt2t;
    t[6] = 1.0;
    t[7] = (double)(int)(sc->dtkey & 0x7fffffffull);
  }
  DT2 = fmin(fmin(DT2, growth * t[4]), dtmx);
  t[3] = 0.5 * (t[1] + DT2);
  t[2] = DT2;
  t[4] = DT2;
  t[0] += DT2;
  t[5] += 1.0;
  sc->dtbits = ~0ull;
  sc->dtkey = ~0ull;
}

__global__ void node_fsky_kernel(int numnod, int nslot, const int* __restrict__ adsky,
                                 const double4* __restrict__ fsky, double* x, double* d, double* v,
                                 const double* __restrict__ ms, const int* __restrict__ icodt, NoallocScalars* sc) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= numnod) return;
  double ax = 0, ay = 0, az = 0;
  const int k0 = max(adsky[n], 0), k1 = min(adsky[n + 1], nslot);   // within the scratch
  for (int k = k0; k < k1; ++k) {
    const double4 f = fsky[k];
    ax += f.x; ay += f.y; az += f.z;
  }
  const double m = ms[n];
  if (m > 0.0) { const double r = 1.0 / m; ax *= r; ay *= r; az *= r; } else { ax = ay = az = 0.0; }
  if (!isfinite(ax + ay + az)) noalloc_error(sc, OR_E_NAN, n);
  double vx = v[3 * n], vy = v[3 * n + 1], vz = v[3 * n + 2];
  const int c = icodt[n];
  if (c & 4) { vx = 0; ax = 0; }
  if (c & 2) { vy = 0; ay = 0; }
  if (c & 1) { vz = 0; az = 0; }
  const double dt12 = sc->time[3], dt2 = sc->time[2];
  vx += dt12 * ax; vy += dt12 * ay; vz += dt12 * az;
  v[3 * n] = vx; v[3 * n + 1] = vy; v[3 * n + 2] = vz;
  const double ux = dt2 * vx, uy = dt2 * vy, uz = dt2 * vz;
  d[3 * n] += ux; d[3 * n + 1] += uy; d[3 * n + 2] += uz;
  x[3 * n] += ux; x[3 * n + 1] += uy; x[3 * n + 2] += uz;
}

__global__ void start_cycle_kernel(NoallocScalars* sc) {
  sc->time[1] = sc->time[2];   // DT1 = DT2 (resol.F:2639)
}

// Bounded wait for the call's own work, as the handle path's wait_stream.
int wait_event(cudaEvent_t ev) {
  double limit = 900.0;
  if (const char* s = std::getenv("OR_ECYCLE_TIMEOUT_S")) limit = std::atof(s);
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t q = cudaEventQuery(ev);
    if (q == cudaSuccess) return OR_OK;
    if (q != cudaErrorNotReady) return OR_E_CUDA;
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > limit) return OR_E_TIMEOUT;
    std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 5 : 200));
  }
}

// Waits (bounded) for the work queued on s, then copies the scalars back.  The
// wait comes first: a copy into pageable host memory blocks until the stream
// drains, so issued before the wait it would make the wait unbounded.
int read_scalars(cudaStream_t s, NoallocScalars* dev, NoallocScalars* out) {
  cudaEvent_t ev;
  if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return OR_E_CUDA;
  const int rc = cudaEventRecord(ev, s) == cudaSuccess ? wait_event(ev) : OR_E_CUDA;
  if (rc == OR_E_TIMEOUT) return rc;        // the work is still running: keep the event
  cudaEventDestroy(ev);
  if (rc) return rc;
  if (cudaMemcpyAsync(out, dev, sizeof *out, cudaMemcpyDeviceToHost, s) != cudaSuccess) return OR_E_CUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? OR_OK : OR_E_CUDA;
}

}  // namespace

extern "C" int or_ecycle_hex_step_noalloc(int device, void* stream, int ncycles, or_ecycle_time* t,
                                          int numnod, double* x, double* d, double* v, const double* ms,
                                          const int* icodt, int nel, const int* conn, const int* iads,
                                          const int* adsky, const or_material* mat, const or_solid_prop* prop,
                                          double dtfac, double dtmx, double dt_growth, double* sig, double* eint,
                                          double* rho, double* qvis, double* pla, double* epsd, const double* vol0) {
  if (!t || !mat || !prop || !x || !d || !v || !ms || !icodt || !conn || !iads || !adsky || !sig || !eint || !rho ||
      !qvis || !pla || !epsd || !vol0)
    return OR_E_ARG;
  if (ncycles < 0 || numnod <= 0 || nel <= 0) return OR_E_ARG;
  if ((long long)8 * nel > OR_NOALLOC_MAX_SLOTS) return OR_E_ARG;       // skyline beyond the scratch
  if (mat->law != OR_LAW_ELASTIC && mat->law != OR_LAW_JOHNSON_COOK) return OR_E_UNSUPPORTED;
  if (prop->jcvt != 0) return OR_E_UNSUPPORTED;                          // global frame only
  if (device < 0 || device >= MAX_DEVICES) return OR_E_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return OR_E_CUDA;
  ScratchPtrs p;
  {
    std::lock_guard<std::mutex> lk(g_ptrs_lock);
    if (!g_ptrs_ready[device]) {
      ScratchPtrs q;
      if (cudaGetSymbolAddress((void**)&q.fsky, g_fsky_scratch) != cudaSuccess) return OR_E_CUDA;
      if (cudaGetSymbolAddress((void**)&q.sc, g_noalloc_scalars) != cudaSuccess) return OR_E_CUDA;
      g_ptrs[device] = q;
      g_ptrs_ready[device] = true;
    }
    p = g_ptrs[device];
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int nslot = 8 * nel;
  // clear what must start at zero / +inf, load the caller's time state
  NoallocScalars init;
  init.dtbits = ~0ull;
  init.dtkey = ~0ull;
  init.err_code = 0;
  init.err_index = -1;
  init.time[0] = t->tt; init.time[1] = t->dt1; init.time[2] = t->dt2; init.time[3] = t->dt12;
  init.time[4] = t->dt2old; init.time[5] = (double)t->ncycle; init.time[6] = (double)t->ityptst;
  init.time[7] = (double)t->neltst;
  if (cudaMemcpyAsync(p.sc, &init, sizeof init, cudaMemcpyHostToDevice, s) != cudaSuccess) return OR_E_CUDA;
  // check the caller's tables before anything is written (slot counters in the scratch)
  NoallocScalars out;
  {
    unsigned* count = reinterpret_cast<unsigned*>(p.fsky);
    if (cudaMemsetAsync(count, 0, (size_t)nslot * sizeof(unsigned), s) != cudaSuccess) return OR_E_CUDA;
    check_adsky_kernel<<<(unsigned)((numnod + 255) / 256), 256, 0, s>>>(nel, numnod, adsky, p.sc);
    check_corners_kernel<<<(unsigned)((nslot + 255) / 256), 256, 0, s>>>(nel, numnod, conn, iads, adsky, count, p.sc);
    if (cudaGetLastError() != cudaSuccess) return OR_E_CUDA;
    const int rc = read_scalars(s, p.sc, &out);
    if (rc) return rc;
    if (out.err_code) { t->neltst = out.err_index; return out.err_code; }
  }
  const unsigned eb = (unsigned)((nel + NOALLOC_TILE - 1) / NOALLOC_TILE);
  const unsigned nb = (unsigned)((numnod + 255) / 256);
  for (int c = 0; c < ncycles; ++c) {
    start_cycle_kernel<<<1, 1, 0, s>>>(p.sc);
    hex_fsky_kernel<<<eb, NOALLOC_TILE, 0, s>>>(nel, conn, iads, x, v, sig, eint, rho, qvis, pla, epsd, vol0, *mat,
                                                 *prop, dtfac, p.fsky, p.sc);
    dt_kernel<<<1, 1, 0, s>>>(p.sc, dt_growth, dtmx);
    node_fsky_kernel<<<nb, 256, 0, s>>>(numnod, nslot, adsky, p.fsky, x, d, v, ms, icodt, p.sc);
  }
  if (cudaGetLastError() != cudaSuccess) return OR_E_CUDA;
  const int rc = read_scalars(s, p.sc, &out);
  if (rc) return rc;
  t->tt = out.time[0]; t->dt1 = out.time[1]; t->dt2 = out.time[2]; t->dt12 = out.time[3];
  t->dt2old = out.time[4]; t->ncycle = (int)out.time[5];
  t->ityptst = (int)out.time[6]; t->neltst = (int)out.time[7];
  if (out.err_code) t->neltst = out.err_index;
  return out.err_code;
}
