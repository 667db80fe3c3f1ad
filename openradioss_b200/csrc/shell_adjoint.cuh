// shell_adjoint.cuh -- reverse mode of one Belytschko-Tsay shell element cycle, FP64.
//
// shell_forward() restates, for one element, the FP64 arithmetic of the shell
// patch kernel (CNVEC3, CDERI3, CDEFO3, CCURV3, CSTRA3, the MULAWC layer loop
// with SIGEPS01C / SIGEPS02C -> M2CPLR IPLA=0, CHVIS3, CFINT3, CUPDT3P signs and
// the uniform pressure load) and records the intermediates in a tape;
// shell_reverse() propagates output adjoints back to the inputs.
//
//   inputs : corner coordinates x, velocities v, rotational velocities vr,
//            per-IP stress sig(5) and plastic strain pla, thickness thk (state),
//            THKE, hourglass history hourg(3), Johnson-Cook A of the element
//   outputs: corner forces f and moments m as assembled into the nodes, the
//            new state (sig, pla, thk, hourg) and the element's plastic work
//
// The time step DT1 is an input constant: the adjoint treats the dt sequence as
// fixed.  CDLEN3 / CDT3 feed only dt and are not differentiated; the element
// energies EINT / EHOU feed no output and are left out.  The radial return is
// differentiated on the branch the forward took (elastic or plastic), the
// clamps (AREA >= 1e-20, THK >= 1e-30, YLD <= SIGMAX) on their active side.
//
// Header-only and free of CUDA types so that it compiles for the host too.
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define ORB_HD __host__ __device__ inline
#else
#define ORB_HD inline
#endif

namespace orb_adj {

constexpr double A_EM15 = 1e-15, A_EM20 = 1e-20, A_EM30 = 1e-30;

struct ShellParams {
  int law, npt, ithk, degen;
  int ishfram, pad;       // local frame: 0, or 2 (/SHFRA/V4, cnvec3.F:82-106)
  double rho, young, nu, shear, a11, a12, jc_b, jc_n, sigmax;
  double hm, hf, hr, shf, pressure;
};

// all-double layouts (no padding), so that flat arrays can stand in for them
template <int NP>
struct ShellIn {
  double x[4][3], v[4][3], vr[4][3];
  double sig[NP][5], pla[NP];
  double thk, thke, hourg[3], ca, dt1;
};

template <int NP>
struct ShellOut {
  double f[4][3], m[4][3];
  double sig[NP][5], pla[NP];
  double thk, hourg[3], wpla;
};

template <int NP>
struct ShellTape {
  double d21[3], d31[3], d41[3], d32[3], d34[3];
  double e1[3], e2[3], e3[3], n3, e3n[3], q1, q2, s, c23[3], e1p[3], n1, e1n[3], e2n[3];
  double e2p[3], n2;      // ISHFRAM 2: e2 before its normalisation
  double X2, Y2, X3, Y3, X4, Y4, PX1, PY1, PX2, PY2, AREA, VHX, VHY;
  int area_clamped;
  double THK0, THK02, GS;
  double VXl[4], VYl[4], VZl[4], RXl[4], RYl[4];
  double VZ13, VZ24, t2a, t1a, t1b, t2b, t3a, t3b, VX13, VX24, VY13, VY24;
  double RX13, RX24, RXAV, RY13, RY24, RYAV;
  double Er[8], E[8], FAC1;   // EXX EYY EXY EYZ EXZ KXX KYY KXY, raw and scaled by DT1/AREA
  double ZT[NP], THKLYL[NP], DXX[NP], DYY[NP], DXY[NP], ST[NP][3], SVM[NP], YLD[NP], RR[NP];
  double DPLA[NP], EZZp[NP], EZZ[NP], SN[NP][5];
  int plastic[NP], yclamp[NP], dpla_pos[NP];
  double FOR[5], MOM[3], THKN;
  double px1v, px2v, py1v, py2v, GAMA[4], T2A, H1Q, H2Q, H3Q, TD, HH1, HH2, B12;
  double A1c, A3c, A5c, A7c, A8c;
  double HG1, HG2, HG3, HG4, HG5, HOUR1A, HOUR2A, HOUR3A, HOUR4, HOUR5;
  double FA[5], Gc[3][3], MA[3], G1m[4], G2m[4], Fg[3][4], Mg[3][4];
  double pa[3], pb[3];
};

ORB_HD void v_cross(const double a[3], const double b[3], double c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
ORB_HD double v_dot(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
// reverse of c = a x b: abar += b x cbar, bbar += cbar x a
ORB_HD void v_cross_rev(const double a[3], const double b[3], const double cb[3], double ab[3], double bb[3]) {
  ab[0] += b[1] * cb[2] - b[2] * cb[1];
  ab[1] += b[2] * cb[0] - b[0] * cb[2];
  ab[2] += b[0] * cb[1] - b[1] * cb[0];
  bb[0] += cb[1] * a[2] - cb[2] * a[1];
  bb[1] += cb[2] * a[0] - cb[0] * a[2];
  bb[2] += cb[0] * a[1] - cb[1] * a[0];
}
// reverse of n = u / max(|u|, 1e-20) given |u| = nu
ORB_HD void v_normalize_rev(const double n[3], double nu, const double nb[3], double ub[3]) {
  if (nu > A_EM20) {
    const double p = v_dot(n, nb);
    for (int c = 0; c < 3; ++c) ub[c] += (nb[c] - n[c] * p) / nu;
  } else {
    for (int c = 0; c < 3; ++c) ub[c] += nb[c] / A_EM20;
  }
}

// ---------------------------------------------------------------------------
// forward
// ---------------------------------------------------------------------------
template <int NP>
ORB_HD void shell_forward(const ShellParams& P, const float* zw, const ShellIn<NP>& in, ShellOut<NP>& out,
                          ShellTape<NP>& t) {
  const double DT1 = in.dt1;
  for (int c = 0; c < 3; ++c) {
    t.d21[c] = in.x[1][c] - in.x[0][c];
    t.d31[c] = in.x[2][c] - in.x[0][c];
    t.d41[c] = in.x[3][c] - in.x[0][c];
    t.d32[c] = in.x[2][c] - in.x[1][c];
    t.d34[c] = in.x[2][c] - in.x[3][c];
  }
  // CNVEC3, ISHFRAM = 0 (cnvec3.F:66-81) or 2 (cnvec3.F:82-106)
  for (int c = 0; c < 3; ++c) { t.e1[c] = t.d21[c] + t.d34[c]; t.e2[c] = t.d32[c] + t.d41[c]; }
  v_cross(t.e1, t.e2, t.e3);
  if (P.ishfram == 2) {
    // e1 = |e2|^2 e1 + e2 x e3 (e3 not normalised), then e1, e3 normalised,
    // e2 = e3 x e1 normalised
    t.q2 = t.e2[0] * t.e2[0] + t.e2[1] * t.e2[1] + t.e2[2] * t.e2[2];
    v_cross(t.e2, t.e3, t.c23);
    for (int c = 0; c < 3; ++c) t.e1p[c] = t.e1[c] * t.q2 + t.c23[c];
    double su = sqrt(t.e1p[0] * t.e1p[0] + t.e1p[1] * t.e1p[1] + t.e1p[2] * t.e1p[2]);
    t.n1 = su;
    su = 1.0 / (su > A_EM20 ? su : A_EM20);
    for (int c = 0; c < 3; ++c) t.e1n[c] = t.e1p[c] * su;
    su = sqrt(t.e3[0] * t.e3[0] + t.e3[1] * t.e3[1] + t.e3[2] * t.e3[2]);
    t.n3 = su;
    su = 1.0 / (su > A_EM20 ? su : A_EM20);
    for (int c = 0; c < 3; ++c) t.e3n[c] = t.e3[c] * su;
    v_cross(t.e3n, t.e1n, t.e2p);
    su = sqrt(t.e2p[0] * t.e2p[0] + t.e2p[1] * t.e2p[1] + t.e2p[2] * t.e2p[2]);
    t.n2 = su;
    su = 1.0 / (su > A_EM20 ? su : A_EM20);
    for (int c = 0; c < 3; ++c) t.e2n[c] = t.e2p[c] * su;
  } else {
    double su = sqrt(t.e3[0] * t.e3[0] + t.e3[1] * t.e3[1] + t.e3[2] * t.e3[2]);
    t.n3 = su;
    su = 1.0 / (su > A_EM20 ? su : A_EM20);
    for (int c = 0; c < 3; ++c) t.e3n[c] = t.e3[c] * su;
    t.q1 = t.e1[0] * t.e1[0] + t.e1[1] * t.e1[1] + t.e1[2] * t.e1[2];
    t.q2 = t.e2[0] * t.e2[0] + t.e2[1] * t.e2[1] + t.e2[2] * t.e2[2];
    t.s = sqrt(t.q1 / t.q2);
    v_cross(t.e2, t.e3n, t.c23);
    for (int c = 0; c < 3; ++c) t.e1p[c] = t.e1[c] + t.c23[c] * t.s;
    su = sqrt(t.e1p[0] * t.e1p[0] + t.e1p[1] * t.e1p[1] + t.e1p[2] * t.e1p[2]);
    t.n1 = su;
    su = 1.0 / (su > A_EM20 ? su : A_EM20);
    for (int c = 0; c < 3; ++c) t.e1n[c] = t.e1p[c] * su;
    v_cross(t.e3n, t.e1n, t.e2n);
  }
  // CDERI3 (cderi3.F:87-190)
  t.X2 = v_dot(t.e1n, t.d21); t.Y2 = v_dot(t.e2n, t.d21);
  t.Y3 = v_dot(t.e2n, t.d31); t.X3 = v_dot(t.e1n, t.d31);
  t.X4 = v_dot(t.e1n, t.d41); t.Y4 = v_dot(t.e2n, t.d41);
  t.PX1 = 0.5 * (t.Y2 - t.Y4); t.PY1 = 0.5 * (t.X4 - t.X2); t.PX2 = 0.5 * t.Y3; t.PY2 = -0.5 * t.X3;
  {
    const double a = 2.0 * (t.PY2 * t.PX1 - t.PY1 * t.PX2);
    t.area_clamped = !(a > A_EM20);
    t.AREA = a > A_EM20 ? a : A_EM20;
  }
  t.VHX = (-t.X2 + t.X3 - t.X4) / t.AREA;
  t.VHY = (-t.Y2 + t.Y3 - t.Y4) / t.AREA;
  // CCOEF3 (ccoef3.F:66-160)
  t.THK0 = P.ithk > 0 ? in.thk : in.thke;
  t.THK02 = t.THK0 * t.THK0;
  const double NU = P.nu, GG = P.shear, YM = P.young;
  const int npt = P.npt;
  const double SHF = npt == 1 ? 0.0 : P.shf;
  t.GS = GG * SHF;
  // CDEFO3, IHBE <= 1 (cdefo3.F:84-131)
  for (int k = 0; k < 4; ++k) {
    t.VXl[k] = v_dot(t.e1n, in.v[k]);
    t.VYl[k] = v_dot(t.e2n, in.v[k]);
    t.VZl[k] = v_dot(t.e3n, in.v[k]);
    t.RXl[k] = v_dot(t.e1n, in.vr[k]);
    t.RYl[k] = v_dot(t.e2n, in.vr[k]);
  }
  const double PX1 = t.PX1, PY1 = t.PY1, PX2 = t.PX2, PY2 = t.PY2;
  double EXX, EYY, EXY, EXZ, EYZ, KXX, KYY, KXY;
  {
    t.VZ13 = t.VZl[0] - t.VZl[2]; t.VZ24 = t.VZl[1] - t.VZl[3];
    EYZ = PY1 * t.VZ13 + PY2 * t.VZ24;
    EXZ = PX1 * t.VZ13 + PX2 * t.VZ24;
    const double DT1V4 = 0.25 * DT1;
    t.t2a = PY2 + PY1;
    t.t3a = copysign(fmax(fabs(t.t2a), A_EM20), t.t2a);
    t.t1a = DT1V4 * (t.VZ13 - t.VZ24) * (t.VZ13 - t.VZ24) / t.t3a;
    t.VX13 = t.VXl[0] - t.VXl[2] - t.t1a; t.VX24 = t.VXl[1] - t.VXl[3] + t.t1a;
    EXX = PX1 * t.VX13 + PX2 * t.VX24;
    EXY = PY1 * t.VX13 + PY2 * t.VX24;
    t.t1b = PX2 - PX1;
    t.t3b = copysign(fmax(fabs(t.t1b), A_EM20), t.t1b);
    t.t2b = DT1V4 * (t.VZ13 + t.VZ24) * (t.VZ13 + t.VZ24) / t.t3b;
    t.VY13 = t.VYl[0] - t.VYl[2] + t.t2b; t.VY24 = t.VYl[1] - t.VYl[3] + t.t2b;
    EXY = EXY + PX1 * t.VY13 + PX2 * t.VY24;
    EYY = PY1 * t.VY13 + PY2 * t.VY24;
    // CCURV3 (ccurv3.F:61-86)
    t.RX13 = t.RXl[0] - t.RXl[2]; t.RXAV = t.RXl[0] + t.RXl[1] + t.RXl[2] + t.RXl[3]; t.RX24 = t.RXl[1] - t.RXl[3];
    KYY = -PY1 * t.RX13 - PY2 * t.RX24;
    const double kxy = PX1 * t.RX13 + PX2 * t.RX24;
    t.RY13 = t.RYl[0] - t.RYl[2]; t.RYAV = t.RYl[0] + t.RYl[1] + t.RYl[2] + t.RYl[3]; t.RY24 = t.RYl[1] - t.RYl[3];
    KXX = PX1 * t.RY13 + PX2 * t.RY24;
    KXY = PY1 * t.RY13 + PY2 * t.RY24 - kxy;
    EXZ = EXZ + t.RYAV * (0.25 * t.AREA);
    EYZ = EYZ - t.RXAV * (0.25 * t.AREA);
  }
  t.Er[0] = EXX; t.Er[1] = EYY; t.Er[2] = EXY; t.Er[3] = EYZ; t.Er[4] = EXZ; t.Er[5] = KXX; t.Er[6] = KYY; t.Er[7] = KXY;
  // CSTRA3 (cstra3.F:91-101)
  t.FAC1 = DT1 / t.AREA;
  for (int i = 0; i < 8; ++i) t.E[i] = t.Er[i] * t.FAC1;
  EXX = t.E[0]; EYY = t.E[1]; EXY = t.E[2]; EYZ = t.E[3]; EXZ = t.E[4]; KXX = t.E[5]; KYY = t.E[6]; KXY = t.E[7];
  // MULAWC layer loop (mulawc.F90:596-1100, 2603-2620)
  const float* Z0 = zw + (npt - 1) * 33;
  const float* WF = Z0 + 11;
  const float* WM = Z0 + 22;
  for (int c = 0; c < 5; ++c) t.FOR[c] = 0.0;
  for (int c = 0; c < 3; ++c) t.MOM[c] = 0.0;
  t.THKN = in.thk;
  const double CA = in.ca, CB = P.jc_b, CN = P.jc_n, YMAX = P.sigmax;
  double wpla = 0.0;
  for (int ip = 0; ip < npt && ip < NP; ++ip) {
    const double wf = (double)WF[ip], wm = (double)WM[ip];
    const double* SO = in.sig[ip];
    double* SN = t.SN[ip];
    t.THKLYL[ip] = wf * t.THK0;
    t.ZT[ip] = (double)Z0[ip] * t.THK0;
    const double DXX = EXX + t.ZT[ip] * KXX, DYY = EYY + t.ZT[ip] * KYY, DXY = EXY + t.ZT[ip] * KXY;
    t.DXX[ip] = DXX; t.DYY[ip] = DYY; t.DXY[ip] = DXY;
    double EZZ = 0.0, PLA = in.pla[ip];
    t.plastic[ip] = 0; t.yclamp[ip] = 0; t.dpla_pos[ip] = 0;
    t.DPLA[ip] = 0.0; t.EZZp[ip] = 0.0; t.SVM[ip] = 0.0; t.YLD[ip] = 0.0; t.RR[ip] = 1.0;
    if (P.law == 1) {
      // SIGEPS01C (sigeps01c.F:130-146)
      SN[0] = SO[0] + P.a11 * DXX + P.a12 * DYY;
      SN[1] = SO[1] + P.a12 * DXX + P.a11 * DYY;
      SN[2] = SO[2] + GG * DXY;
      SN[3] = SO[3] + t.GS * EYZ;
      SN[4] = SO[4] + t.GS * EXZ;
      EZZ = -NU * (DXX + DYY) / (1.0 - NU);
    } else {
      // SIGEPS02C -> M2CPLR, IPLA = 0 (m2cplr.F:96-230)
      const double A1 = YM / (1.0 - NU * NU), A2 = A1 * NU;
      SN[0] = SO[0] + A1 * DXX + A2 * DYY;
      SN[1] = SO[1] + A2 * DXX + A1 * DYY;
      SN[2] = SO[2] + GG * DXY;
      SN[3] = SO[3] + t.GS * EYZ;
      SN[4] = SO[4] + t.GS * EXZ;
      t.ST[ip][0] = SN[0]; t.ST[ip][1] = SN[1]; t.ST[ip][2] = SN[2];
      double YLD = PLA == 0.0 ? CA : CA + CB * exp(CN * log(PLA));
      t.yclamp[ip] = YLD > YMAX;
      YLD = fmin(YLD, YMAX);
      const double SVM = sqrt(SN[0] * SN[0] + SN[1] * SN[1] - SN[0] * SN[1] + 3.0 * SN[2] * SN[2]);
      const double RR = fmin(1.0, YLD / (SVM + A_EM15));
      double DPLA = 0.0, EZZp = 0.0;
      if (RR < 1.0) {
        t.plastic[ip] = 1;
        SN[0] *= RR; SN[1] *= RR; SN[2] *= RR;
        const double q = (SVM - YLD) / YM;
        t.dpla_pos[ip] = q > 0.0;
        DPLA = fmax(0.0, q);
        EZZp = DPLA * (0.5 * (SN[0] + SN[1])) / YLD;
        PLA = PLA + DPLA;
      }
      EZZ = -(DXX + DYY) * NU - (1.0 - 2.0 * NU) * EZZp;   // sigeps02c.F:215-224
      EZZ = EZZ / (1.0 - NU);
      wpla += YLD * DPLA * t.AREA * t.THKLYL[ip];
      t.SVM[ip] = SVM; t.YLD[ip] = YLD; t.RR[ip] = RR; t.DPLA[ip] = DPLA; t.EZZp[ip] = EZZp;
    }
    t.EZZ[ip] = EZZ;
    t.THKN = t.THKN + EZZ * t.THKLYL[ip];
    for (int c = 0; c < 5; ++c) { out.sig[ip][c] = SN[c]; t.FOR[c] = t.FOR[c] + wf * SN[c]; }
    for (int c = 0; c < 3; ++c) t.MOM[c] = t.MOM[c] + wm * SN[c];
    out.pla[ip] = PLA;
  }
  out.wpla = wpla;
  out.thk = t.THKN > A_EM30 ? t.THKN : A_EM30;
  // CHVIS3, ISMSTR = 2, IHBE = 1, HELAS = HVISC = 1/2, HVLIN = 0 (chvis3.F:116-300)
  {
    t.px1v = PX1 * t.VHX; t.px2v = PX2 * t.VHX; t.py1v = PY1 * t.VHY; t.py2v = PY2 * t.VHY;
    t.GAMA[0] = 1.0 - t.px1v - t.py1v;
    t.GAMA[2] = 1.0 + t.px1v + t.py1v;
    t.GAMA[1] = -1.0 - t.px2v - t.py2v;
    t.GAMA[3] = -1.0 + t.px2v + t.py2v;
    const double SHFPR3 = SHF / (3.0 * (1.0 + NU));
    const double R1 = 0.25 * P.rho * 100.0;
    t.A1c = R1 * (0.5 * P.hm);
    t.A3c = R1 * (0.5 * P.hf) * sqrt(SHFPR3);
    t.A5c = 0.5 * P.hr * R1 * 0.072169;
    const double R0e = 0.25 * YM * 0.5;
    t.A7c = P.hm * R0e; t.A8c = P.hf * R0e * SHFPR3;
    t.T2A = t.THK02 * t.AREA;
    t.H1Q = t.A1c * sqrt(t.T2A); t.H2Q = t.A3c * t.THK02; t.H3Q = t.A5c * t.T2A;
    t.TD = t.THK0 * DT1;
    t.HH1 = t.A7c * t.TD;
    const double B1 = PX1 * PX1 + PY1 * PY1, B2 = PX2 * PX2 + PY2 * PY2;
    t.B12 = B1 + B2;
    t.HH2 = t.A8c * t.THK02 * t.TD / t.B12;
    if (P.degen) { t.H1Q = t.H2Q = t.H3Q = t.HH1 = t.HH2 = 0.0; }
    t.HG1 = t.VXl[0] * t.GAMA[0] + t.VXl[1] * t.GAMA[1] + t.VXl[2] * t.GAMA[2] + t.VXl[3] * t.GAMA[3];
    t.HG2 = t.VYl[0] * t.GAMA[0] + t.VYl[1] * t.GAMA[1] + t.VYl[2] * t.GAMA[2] + t.VYl[3] * t.GAMA[3];
    const double hour1 = in.hourg[0] + t.HG1 * t.HH1;
    const double hour2 = in.hourg[1] + t.HG2 * t.HH1;
    t.HOUR1A = hour1 + t.HG1 * (t.H1Q * fabs(t.HG1));
    t.HOUR2A = hour2 + t.HG2 * (t.H1Q * fabs(t.HG2));
    t.HG3 = t.VZl[0] * t.GAMA[0] + t.VZl[1] * t.GAMA[1] + t.VZl[2] * t.GAMA[2] + t.VZl[3] * t.GAMA[3];
    const double hour3 = in.hourg[2] + t.HG3 * t.HH2;
    t.HOUR3A = hour3 + t.HG3 * (t.H2Q * fabs(t.HG3));
    t.HG4 = t.RXl[0] - t.RXl[1] + t.RXl[2] - t.RXl[3];
    t.HG5 = t.RYl[0] - t.RYl[1] + t.RYl[2] - t.RYl[3];
    t.HOUR4 = t.HG4 * (t.H3Q * fabs(t.HG4));
    t.HOUR5 = t.HG5 * (t.H3Q * fabs(t.HG5));
    out.hourg[0] = hour1; out.hourg[1] = hour2; out.hourg[2] = hour3;
  }
  // CFINT3, ISIGI = 0 (cfint3.F:173-260)
  {
    for (int c = 0; c < 5; ++c) t.FA[c] = t.FOR[c] * t.THK0;
    const double F1A = t.FA[0], F2A = t.FA[1], F3A = t.FA[2], F4A = t.FA[3], F5A = t.FA[4];
    const double M4 = 0.25 * (F4A * t.AREA), M5 = 0.25 * (F5A * t.AREA);
    const double F12 = F1A * PX2 + F3A * PY2, F22 = F2A * PY2 + F3A * PX2, F32 = F5A * PX2 + F4A * PY2;
    const double F11 = F1A * PX1 + F3A * PY1, F21 = F2A * PY1 + F3A * PX1, F31 = F5A * PX1 + F4A * PY1;
    double H1j[3], H2j[3], H3j[3];
    for (int k = 0; k < 3; ++k) { H1j[k] = t.HOUR1A * t.GAMA[k]; H2j[k] = t.HOUR2A * t.GAMA[k]; H3j[k] = t.HOUR3A * t.GAMA[k]; }
    t.Gc[0][0] = F11 + H1j[0]; t.Gc[0][1] = F12 + H1j[1]; t.Gc[0][2] = H1j[2] - F11;
    t.Gc[1][0] = F21 + H2j[0]; t.Gc[1][1] = F22 + H2j[1]; t.Gc[1][2] = H2j[2] - F21;
    t.Gc[2][0] = F31 + H3j[0]; t.Gc[2][1] = F32 + H3j[1]; t.Gc[2][2] = H3j[2] - F31;
    for (int k = 0; k < 3; ++k)
      for (int c = 0; c < 3; ++c)
        t.Fg[c][k] = t.e1n[c] * t.Gc[0][k] + t.e2n[c] * t.Gc[1][k] + t.e3n[c] * t.Gc[2][k];
    for (int c = 0; c < 3; ++c) t.Fg[c][3] = -t.Fg[c][0] - t.Fg[c][1] - t.Fg[c][2];
    for (int c = 0; c < 3; ++c) t.MA[c] = t.MOM[c] * t.THK02;
    const double M1A = t.MA[0], M2A = t.MA[1], M3A = t.MA[2];
    const double M11 = -M2A * PY1 - M3A * PX1, M21 = M1A * PX1 + M3A * PY1;
    const double M12 = -M2A * PY2 - M3A * PX2, M22 = M1A * PX2 + M3A * PY2;
    t.G1m[0] = M11 - M4 + t.HOUR4; t.G1m[1] = M12 - M4 - t.HOUR4; t.G1m[2] = -M11 - M4 + t.HOUR4; t.G1m[3] = -M12 - M4 - t.HOUR4;
    t.G2m[0] = M21 + M5 + t.HOUR5; t.G2m[1] = M22 + M5 - t.HOUR5; t.G2m[2] = -M21 + M5 + t.HOUR5; t.G2m[3] = -M22 + M5 - t.HOUR5;
    for (int k = 0; k < 4; ++k)
      for (int c = 0; c < 3; ++c) t.Mg[c][k] = t.e1n[c] * t.G1m[k] + t.e2n[c] * t.G2m[k];
  }
  // uniform pressure (load_pressure.F:201-207): F = -p N / 8, N = x13 x x24
  double PF[3] = {0.0, 0.0, 0.0};
  for (int c = 0; c < 3; ++c) { t.pa[c] = in.x[2][c] - in.x[0][c]; t.pb[c] = in.x[3][c] - in.x[1][c]; }
  if (P.pressure != 0.0) {
    double N[3];
    v_cross(t.pa, t.pb, N);
    const double AA = -P.pressure * 0.125;
    for (int c = 0; c < 3; ++c) PF[c] = AA * N[c];
  }
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) { out.f[k][c] = -t.Fg[c][k] + PF[c]; out.m[k][c] = -t.Mg[c][k]; }
}

// ---------------------------------------------------------------------------
// reverse: ob = adjoints of the outputs, ib = adjoints of the inputs (accumulated)
// ---------------------------------------------------------------------------
template <int NP>
ORB_HD void shell_reverse(const ShellParams& P, const float* zw, const ShellIn<NP>& in, const ShellTape<NP>& t,
                          const ShellOut<NP>& ob, ShellIn<NP>& ib) {
  const double DT1 = in.dt1;
  const double NU = P.nu, GG = P.shear, YM = P.young;
  const int npt = P.npt;
  const double PX1 = t.PX1, PY1 = t.PY1, PX2 = t.PX2, PY2 = t.PY2;
  double bPX1 = 0, bPY1 = 0, bPX2 = 0, bPY2 = 0, bAREA = 0, bTHK0 = 0, bTHK02 = 0, bVHX = 0, bVHY = 0;
  double be1n[3] = {0, 0, 0}, be2n[3] = {0, 0, 0}, be3n[3] = {0, 0, 0};
  double bVXl[4] = {0, 0, 0, 0}, bVYl[4] = {0, 0, 0, 0}, bVZl[4] = {0, 0, 0, 0}, bRXl[4] = {0, 0, 0, 0},
         bRYl[4] = {0, 0, 0, 0};
  // ---- outputs f, m ----
  double bFg[3][4], bMg[3][4], bPF[3] = {0, 0, 0};
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) {
      bFg[c][k] = -ob.f[k][c];
      bPF[c] += ob.f[k][c];
      bMg[c][k] = -ob.m[k][c];
    }
  // ---- pressure ----
  if (P.pressure != 0.0) {
    const double AA = -P.pressure * 0.125;
    double bN[3] = {AA * bPF[0], AA * bPF[1], AA * bPF[2]}, bpa[3] = {0, 0, 0}, bpb[3] = {0, 0, 0};
    v_cross_rev(t.pa, t.pb, bN, bpa, bpb);
    for (int c = 0; c < 3; ++c) {
      ib.x[2][c] += bpa[c]; ib.x[0][c] -= bpa[c];
      ib.x[3][c] += bpb[c]; ib.x[1][c] -= bpb[c];
    }
  }
  // ---- CFINT3 moments ----
  double bG1m[4] = {0, 0, 0, 0}, bG2m[4] = {0, 0, 0, 0};
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) {
      be1n[c] += bMg[c][k] * t.G1m[k];
      be2n[c] += bMg[c][k] * t.G2m[k];
      bG1m[k] += bMg[c][k] * t.e1n[c];
      bG2m[k] += bMg[c][k] * t.e2n[c];
    }
  const double bM11 = bG1m[0] - bG1m[2], bM12 = bG1m[1] - bG1m[3];
  const double bM21 = bG2m[0] - bG2m[2], bM22 = bG2m[1] - bG2m[3];
  const double bM4 = -(bG1m[0] + bG1m[1] + bG1m[2] + bG1m[3]);
  const double bM5 = bG2m[0] + bG2m[1] + bG2m[2] + bG2m[3];
  const double bHOUR4 = bG1m[0] - bG1m[1] + bG1m[2] - bG1m[3];
  const double bHOUR5 = bG2m[0] - bG2m[1] + bG2m[2] - bG2m[3];
  const double M1A = t.MA[0], M2A = t.MA[1], M3A = t.MA[2];
  double bMA[3] = {0, 0, 0};
  // M11 = -M2A*PY1 - M3A*PX1 ; M21 = M1A*PX1 + M3A*PY1 ; M12 = -M2A*PY2 - M3A*PX2 ; M22 = M1A*PX2 + M3A*PY2
  bMA[1] -= bM11 * PY1; bPY1 -= bM11 * M2A; bMA[2] -= bM11 * PX1; bPX1 -= bM11 * M3A;
  bMA[0] += bM21 * PX1; bPX1 += bM21 * M1A; bMA[2] += bM21 * PY1; bPY1 += bM21 * M3A;
  bMA[1] -= bM12 * PY2; bPY2 -= bM12 * M2A; bMA[2] -= bM12 * PX2; bPX2 -= bM12 * M3A;
  bMA[0] += bM22 * PX2; bPX2 += bM22 * M1A; bMA[2] += bM22 * PY2; bPY2 += bM22 * M3A;
  double bMOM[3];
  for (int c = 0; c < 3; ++c) { bMOM[c] = bMA[c] * t.THK02; bTHK02 += bMA[c] * t.MOM[c]; }
  // ---- CFINT3 forces ----
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < 3; ++k) bFg[c][k] -= bFg[c][3];
  double bGc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) {
      be1n[c] += bFg[c][k] * t.Gc[0][k];
      be2n[c] += bFg[c][k] * t.Gc[1][k];
      be3n[c] += bFg[c][k] * t.Gc[2][k];
      bGc[0][k] += bFg[c][k] * t.e1n[c];
      bGc[1][k] += bFg[c][k] * t.e2n[c];
      bGc[2][k] += bFg[c][k] * t.e3n[c];
    }
  const double bF11 = bGc[0][0] - bGc[0][2], bF12 = bGc[0][1];
  const double bF21 = bGc[1][0] - bGc[1][2], bF22 = bGc[1][1];
  const double bF31 = bGc[2][0] - bGc[2][2], bF32 = bGc[2][1];
  double bH1j[3] = {bGc[0][0], bGc[0][1], bGc[0][2]};
  double bH2j[3] = {bGc[1][0], bGc[1][1], bGc[1][2]};
  double bH3j[3] = {bGc[2][0], bGc[2][1], bGc[2][2]};
  const double F1A = t.FA[0], F2A = t.FA[1], F3A = t.FA[2], F4A = t.FA[3], F5A = t.FA[4];
  double bFA[5] = {0, 0, 0, 0, 0};
  // F11 = F1A*PX1 + F3A*PY1 ; F21 = F2A*PY1 + F3A*PX1 ; F31 = F5A*PX1 + F4A*PY1
  bFA[0] += bF11 * PX1; bPX1 += bF11 * F1A; bFA[2] += bF11 * PY1; bPY1 += bF11 * F3A;
  bFA[1] += bF21 * PY1; bPY1 += bF21 * F2A; bFA[2] += bF21 * PX1; bPX1 += bF21 * F3A;
  bFA[4] += bF31 * PX1; bPX1 += bF31 * F5A; bFA[3] += bF31 * PY1; bPY1 += bF31 * F4A;
  // F12 = F1A*PX2 + F3A*PY2 ; F22 = F2A*PY2 + F3A*PX2 ; F32 = F5A*PX2 + F4A*PY2
  bFA[0] += bF12 * PX2; bPX2 += bF12 * F1A; bFA[2] += bF12 * PY2; bPY2 += bF12 * F3A;
  bFA[1] += bF22 * PY2; bPY2 += bF22 * F2A; bFA[2] += bF22 * PX2; bPX2 += bF22 * F3A;
  bFA[4] += bF32 * PX2; bPX2 += bF32 * F5A; bFA[3] += bF32 * PY2; bPY2 += bF32 * F4A;
  // M4 = 0.25*F4A*AREA ; M5 = 0.25*F5A*AREA
  bFA[3] += 0.25 * bM4 * t.AREA; bAREA += 0.25 * bM4 * F4A;
  bFA[4] += 0.25 * bM5 * t.AREA; bAREA += 0.25 * bM5 * F5A;
  double bFOR[5];
  for (int c = 0; c < 5; ++c) { bFOR[c] = bFA[c] * t.THK0; bTHK0 += bFA[c] * t.FOR[c]; }
  // ---- CHVIS3 ----
  double bGAMA[4] = {0, 0, 0, 0};
  double bHOUR1A = 0, bHOUR2A = 0, bHOUR3A = 0;
  for (int k = 0; k < 3; ++k) {
    bHOUR1A += bH1j[k] * t.GAMA[k]; bGAMA[k] += bH1j[k] * t.HOUR1A;
    bHOUR2A += bH2j[k] * t.GAMA[k]; bGAMA[k] += bH2j[k] * t.HOUR2A;
    bHOUR3A += bH3j[k] * t.GAMA[k]; bGAMA[k] += bH3j[k] * t.HOUR3A;
  }
  double bH1Q = 0, bH2Q = 0, bH3Q = 0, bHH1 = 0, bHH2 = 0;
  // HOUR4 = HG4*H3Q*|HG4| ; HOUR5 = HG5*H3Q*|HG5|
  const double bHG4 = bHOUR4 * 2.0 * t.H3Q * fabs(t.HG4);
  const double bHG5 = bHOUR5 * 2.0 * t.H3Q * fabs(t.HG5);
  bH3Q += bHOUR4 * t.HG4 * fabs(t.HG4) + bHOUR5 * t.HG5 * fabs(t.HG5);
  bRXl[0] += bHG4; bRXl[1] -= bHG4; bRXl[2] += bHG4; bRXl[3] -= bHG4;
  bRYl[0] += bHG5; bRYl[1] -= bHG5; bRYl[2] += bHG5; bRYl[3] -= bHG5;
  // HOUR3A = hour3 + HG3*H2Q*|HG3| ; hour3 = h2 + HG3*HH2 (hour3 is also the output state)
  {
    const double bhour3 = bHOUR3A + ob.hourg[2];
    double bHG3 = bHOUR3A * 2.0 * t.H2Q * fabs(t.HG3) + bhour3 * t.HH2;
    bH2Q += bHOUR3A * t.HG3 * fabs(t.HG3);
    bHH2 += bhour3 * t.HG3;
    ib.hourg[2] += bhour3;
    for (int k = 0; k < 4; ++k) { bVZl[k] += bHG3 * t.GAMA[k]; bGAMA[k] += bHG3 * t.VZl[k]; }
  }
  {
    const double bhour1 = bHOUR1A + ob.hourg[0];
    const double bhour2 = bHOUR2A + ob.hourg[1];
    const double bHG1 = bHOUR1A * 2.0 * t.H1Q * fabs(t.HG1) + bhour1 * t.HH1;
    const double bHG2 = bHOUR2A * 2.0 * t.H1Q * fabs(t.HG2) + bhour2 * t.HH1;
    bH1Q += bHOUR1A * t.HG1 * fabs(t.HG1) + bHOUR2A * t.HG2 * fabs(t.HG2);
    bHH1 += bhour1 * t.HG1 + bhour2 * t.HG2;
    ib.hourg[0] += bhour1;
    ib.hourg[1] += bhour2;
    for (int k = 0; k < 4; ++k) {
      bVXl[k] += bHG1 * t.GAMA[k]; bVYl[k] += bHG2 * t.GAMA[k];
      bGAMA[k] += bHG1 * t.VXl[k] + bHG2 * t.VYl[k];
    }
  }
  if (!P.degen) {
    // HH2 = A8c*THK02*TD/B12 ; HH1 = A7c*TD ; H3Q = A5c*T2A ; H2Q = A3c*THK02 ; H1Q = A1c*sqrt(T2A)
    double bTD = bHH2 * t.A8c * t.THK02 / t.B12 + bHH1 * t.A7c;
    bTHK02 += bHH2 * t.A8c * t.TD / t.B12;
    const double bB12 = -bHH2 * t.HH2 / t.B12;
    bPX1 += 2.0 * bB12 * PX1; bPY1 += 2.0 * bB12 * PY1; bPX2 += 2.0 * bB12 * PX2; bPY2 += 2.0 * bB12 * PY2;
    double bT2A = bH3Q * t.A5c;
    bTHK02 += bH2Q * t.A3c;
    if (t.T2A > 0.0) bT2A += bH1Q * t.A1c * 0.5 / sqrt(t.T2A);
    bTHK0 += bTD * DT1;
    bTHK02 += bT2A * t.AREA;
    bAREA += bT2A * t.THK02;
  }
  // GAMA
  {
    const double bpx1v = -bGAMA[0] + bGAMA[2], bpy1v = bpx1v;
    const double bpx2v = -bGAMA[1] + bGAMA[3], bpy2v = bpx2v;
    bPX1 += bpx1v * t.VHX; bVHX += bpx1v * PX1;
    bPX2 += bpx2v * t.VHX; bVHX += bpx2v * PX2;
    bPY1 += bpy1v * t.VHY; bVHY += bpy1v * PY1;
    bPY2 += bpy2v * t.VHY; bVHY += bpy2v * PY2;
  }
  // ---- MULAWC layer loop ----
  double bE[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  {
    const double bTHKN = t.THKN > A_EM30 ? ob.thk : 0.0;
    ib.thk += bTHKN;
    const float* Z0 = zw + (npt - 1) * 33;
    const float* WF = Z0 + 11;
    const float* WM = Z0 + 22;
    const double CB = P.jc_b, CN = P.jc_n;
    const double bwpla = ob.wpla;
    for (int ip = 0; ip < npt && ip < NP; ++ip) {
      const double wf = (double)WF[ip], wm = (double)WM[ip];
      double bSN[5];
      for (int c = 0; c < 5; ++c) bSN[c] = ob.sig[ip][c] + wf * bFOR[c];
      for (int c = 0; c < 3; ++c) bSN[c] += wm * bMOM[c];
      double bEZZ = bTHKN * t.THKLYL[ip];
      double bTHKLYL = bTHKN * t.EZZ[ip];
      double bDXX = 0, bDYY = 0, bDXY = 0;
      if (P.law == 1) {
        bDXX += -NU / (1.0 - NU) * bEZZ; bDYY += -NU / (1.0 - NU) * bEZZ;
        for (int c = 0; c < 5; ++c) ib.sig[ip][c] += bSN[c];
        bDXX += P.a11 * bSN[0] + P.a12 * bSN[1];
        bDYY += P.a12 * bSN[0] + P.a11 * bSN[1];
        bDXY += GG * bSN[2];
        bE[3] += t.GS * bSN[3];
        bE[4] += t.GS * bSN[4];
        ib.pla[ip] += ob.pla[ip];
      } else {
        const double A1 = YM / (1.0 - NU * NU), A2 = A1 * NU;
        const double YLD = t.YLD[ip], DPLA = t.DPLA[ip], SVM = t.SVM[ip], RR = t.RR[ip];
        // wpla += YLD*DPLA*AREA*THKLYL
        double bYLD = bwpla * DPLA * t.AREA * t.THKLYL[ip];
        double bDPLA = bwpla * YLD * t.AREA * t.THKLYL[ip];
        bAREA += bwpla * YLD * DPLA * t.THKLYL[ip];
        bTHKLYL += bwpla * YLD * DPLA * t.AREA;
        // EZZ = (-(DXX+DYY)*NU - (1-2NU)*EZZp) / (1-NU)
        bDXX += -NU / (1.0 - NU) * bEZZ; bDYY += -NU / (1.0 - NU) * bEZZ;
        const double bEZZp = -(1.0 - 2.0 * NU) / (1.0 - NU) * bEZZ;
        // PLA_out = PLA_in + DPLA
        ib.pla[ip] += ob.pla[ip];
        double bST[3] = {bSN[0], bSN[1], bSN[2]};
        if (t.plastic[ip]) {
          bDPLA += ob.pla[ip];
          // EZZp = DPLA*0.5*(SN0+SN1)/YLD, SN scaled
          const double SN0 = t.SN[ip][0], SN1 = t.SN[ip][1];
          bDPLA += bEZZp * 0.5 * (SN0 + SN1) / YLD;
          const double bs01 = bEZZp * DPLA * 0.5 / YLD;
          double bSNs[3] = {bSN[0] + bs01, bSN[1] + bs01, bSN[2]};
          bYLD += -bEZZp * t.EZZp[ip] / YLD;
          // DPLA = max(0, (SVM - YLD)/YM)
          double bSVM = 0.0;
          if (t.dpla_pos[ip]) { bSVM += bDPLA / YM; bYLD -= bDPLA / YM; }
          // SN[i] = RR*ST[i], i < 3
          double bRR = 0.0;
          for (int i = 0; i < 3; ++i) { bRR += bSNs[i] * t.ST[ip][i]; bST[i] = bSNs[i] * RR; }
          // RR = YLD/(SVM + EM15)
          const double den = SVM + A_EM15;
          bYLD += bRR / den;
          bSVM -= bRR * YLD / (den * den);
          // SVM = sqrt(S0^2 + S1^2 - S0 S1 + 3 S2^2) of the trial stress
          if (SVM > 0.0) {
            const double bQ = bSVM / (2.0 * SVM);
            const double S0 = t.ST[ip][0], S1 = t.ST[ip][1], S2 = t.ST[ip][2];
            bST[0] += bQ * (2.0 * S0 - S1);
            bST[1] += bQ * (2.0 * S1 - S0);
            bST[2] += bQ * 6.0 * S2;
          }
        }
        // YLD = min(CA + CB*PLA^CN, YMAX), CA when PLA == 0
        if (!t.yclamp[ip]) {
          ib.ca += bYLD;
          const double PLA = in.pla[ip];
          if (PLA > 0.0) ib.pla[ip] += bYLD * CB * CN * exp((CN - 1.0) * log(PLA));
        }
        // trial stress
        for (int c = 0; c < 3; ++c) ib.sig[ip][c] += bST[c];
        ib.sig[ip][3] += bSN[3];
        ib.sig[ip][4] += bSN[4];
        bDXX += A1 * bST[0] + A2 * bST[1];
        bDYY += A2 * bST[0] + A1 * bST[1];
        bDXY += GG * bST[2];
        bE[3] += t.GS * bSN[3];
        bE[4] += t.GS * bSN[4];
      }
      // DXX = EXX + ZT*KXX ...
      bE[0] += bDXX; bE[5] += t.ZT[ip] * bDXX;
      bE[1] += bDYY; bE[6] += t.ZT[ip] * bDYY;
      bE[2] += bDXY; bE[7] += t.ZT[ip] * bDXY;
      const double bZT = bDXX * t.E[5] + bDYY * t.E[6] + bDXY * t.E[7];
      bTHK0 += (double)Z0[ip] * bZT + wf * bTHKLYL;
    }
  }
  // ---- CSTRA3 ----
  double bEr[8];
  {
    double bFAC1 = 0.0;
    for (int i = 0; i < 8; ++i) { bEr[i] = bE[i] * t.FAC1; bFAC1 += bE[i] * t.Er[i]; }
    bAREA -= bFAC1 * t.FAC1 / t.AREA;
  }
  // ---- CCURV3 ----
  // EXZ += RYAV*0.25*AREA ; EYZ -= RXAV*0.25*AREA
  const double bRYAV = bEr[4] * 0.25 * t.AREA, bRXAV = -bEr[3] * 0.25 * t.AREA;
  bAREA += 0.25 * (bEr[4] * t.RYAV - bEr[3] * t.RXAV);
  {
    // KXX = PX1*RY13 + PX2*RY24 ; KXY = PY1*RY13 + PY2*RY24 - kxy ; kxy = PX1*RX13 + PX2*RX24
    // KYY = -PY1*RX13 - PY2*RX24
    const double bKXX = bEr[5], bKYY = bEr[6], bKXY = bEr[7], bkxy = -bKXY;
    const double bRY13 = bKXX * PX1 + bKXY * PY1, bRY24 = bKXX * PX2 + bKXY * PY2;
    bPX1 += bKXX * t.RY13; bPX2 += bKXX * t.RY24; bPY1 += bKXY * t.RY13; bPY2 += bKXY * t.RY24;
    const double bRX13 = bkxy * PX1 - bKYY * PY1, bRX24 = bkxy * PX2 - bKYY * PY2;
    bPX1 += bkxy * t.RX13; bPX2 += bkxy * t.RX24; bPY1 -= bKYY * t.RX13; bPY2 -= bKYY * t.RX24;
    bRXl[0] += bRX13 + bRXAV; bRXl[1] += bRX24 + bRXAV; bRXl[2] += -bRX13 + bRXAV; bRXl[3] += -bRX24 + bRXAV;
    bRYl[0] += bRY13 + bRYAV; bRYl[1] += bRY24 + bRYAV; bRYl[2] += -bRY13 + bRYAV; bRYl[3] += -bRY24 + bRYAV;
  }
  // ---- CDEFO3 ----
  {
    const double bEXX = bEr[0], bEYY = bEr[1], bEXY = bEr[2], bEYZ = bEr[3], bEXZ = bEr[4];
    const double DT1V4 = 0.25 * DT1;
    // EYY = PY1*VY13 + PY2*VY24 ; EXY += PX1*VY13 + PX2*VY24
    const double bVY13 = bEYY * PY1 + bEXY * PX1, bVY24 = bEYY * PY2 + bEXY * PX2;
    bPY1 += bEYY * t.VY13; bPY2 += bEYY * t.VY24; bPX1 += bEXY * t.VY13; bPX2 += bEXY * t.VY24;
    // VY13 = VYl0 - VYl2 + t2b ; VY24 = VYl1 - VYl3 + t2b
    bVYl[0] += bVY13; bVYl[2] -= bVY13; bVYl[1] += bVY24; bVYl[3] -= bVY24;
    const double bt2b = bVY13 + bVY24;
    // t2b = DT1V4*(VZ13+VZ24)^2 / t3b ; t3b = t1b = PX2 - PX1 when |t1b| > 1e-20
    const double sZ = t.VZ13 + t.VZ24;
    double bVZ13 = bt2b * DT1V4 * 2.0 * sZ / t.t3b, bVZ24 = bVZ13;
    if (fabs(t.t1b) > A_EM20) {
      const double bt1b = -bt2b * t.t2b / t.t3b;
      bPX2 += bt1b; bPX1 -= bt1b;
    }
    // EXX = PX1*VX13 + PX2*VX24 ; EXY = PY1*VX13 + PY2*VX24
    const double bVX13 = bEXX * PX1 + bEXY * PY1, bVX24 = bEXX * PX2 + bEXY * PY2;
    bPX1 += bEXX * t.VX13; bPX2 += bEXX * t.VX24; bPY1 += bEXY * t.VX13; bPY2 += bEXY * t.VX24;
    // VX13 = VXl0 - VXl2 - t1a ; VX24 = VXl1 - VXl3 + t1a
    bVXl[0] += bVX13; bVXl[2] -= bVX13; bVXl[1] += bVX24; bVXl[3] -= bVX24;
    const double bt1a = -bVX13 + bVX24;
    // t1a = DT1V4*(VZ13-VZ24)^2 / t3a ; t3a = t2a = PY2 + PY1
    const double dZ = t.VZ13 - t.VZ24;
    const double g = bt1a * DT1V4 * 2.0 * dZ / t.t3a;
    bVZ13 += g; bVZ24 -= g;
    if (fabs(t.t2a) > A_EM20) {
      const double bt2a = -bt1a * t.t1a / t.t3a;
      bPY2 += bt2a; bPY1 += bt2a;
    }
    // EYZ = PY1*VZ13 + PY2*VZ24 ; EXZ = PX1*VZ13 + PX2*VZ24
    bVZ13 += bEYZ * PY1 + bEXZ * PX1; bVZ24 += bEYZ * PY2 + bEXZ * PX2;
    bPY1 += bEYZ * t.VZ13; bPY2 += bEYZ * t.VZ24; bPX1 += bEXZ * t.VZ13; bPX2 += bEXZ * t.VZ24;
    bVZl[0] += bVZ13; bVZl[2] -= bVZ13; bVZl[1] += bVZ24; bVZl[3] -= bVZ24;
  }
  // local velocities: VXl = e1n.v, VYl = e2n.v, VZl = e3n.v, RXl = e1n.vr, RYl = e2n.vr
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) {
      be1n[c] += bVXl[k] * in.v[k][c] + bRXl[k] * in.vr[k][c];
      be2n[c] += bVYl[k] * in.v[k][c] + bRYl[k] * in.vr[k][c];
      be3n[c] += bVZl[k] * in.v[k][c];
      ib.v[k][c] += bVXl[k] * t.e1n[c] + bVYl[k] * t.e2n[c] + bVZl[k] * t.e3n[c];
      ib.vr[k][c] += bRXl[k] * t.e1n[c] + bRYl[k] * t.e2n[c];
    }
  // ---- CCOEF3: THK0, THK02 ----
  bTHK0 += 2.0 * t.THK0 * bTHK02;
  if (P.ithk > 0) ib.thk += bTHK0; else ib.thke += bTHK0;
  // ---- CDERI3 ----
  double bX2 = 0, bY2 = 0, bX3 = 0, bY3 = 0, bX4 = 0, bY4 = 0;
  // VHX = (-X2 + X3 - X4)/AREA ; VHY = (-Y2 + Y3 - Y4)/AREA
  bX2 -= bVHX / t.AREA; bX3 += bVHX / t.AREA; bX4 -= bVHX / t.AREA; bAREA -= bVHX * t.VHX / t.AREA;
  bY2 -= bVHY / t.AREA; bY3 += bVHY / t.AREA; bY4 -= bVHY / t.AREA; bAREA -= bVHY * t.VHY / t.AREA;
  if (!t.area_clamped) {
    // AREA = 2*(PY2*PX1 - PY1*PX2)
    bPY2 += 2.0 * bAREA * PX1; bPX1 += 2.0 * bAREA * PY2;
    bPY1 -= 2.0 * bAREA * PX2; bPX2 -= 2.0 * bAREA * PY1;
  }
  // PX1 = (Y2-Y4)/2 ; PY1 = (X4-X2)/2 ; PX2 = Y3/2 ; PY2 = -X3/2
  bY2 += 0.5 * bPX1; bY4 -= 0.5 * bPX1;
  bX4 += 0.5 * bPY1; bX2 -= 0.5 * bPY1;
  bY3 += 0.5 * bPX2;
  bX3 -= 0.5 * bPY2;
  double bd21[3], bd31[3], bd41[3], bd32[3] = {0, 0, 0}, bd34[3] = {0, 0, 0};
  for (int c = 0; c < 3; ++c) {
    be1n[c] += bX2 * t.d21[c] + bX3 * t.d31[c] + bX4 * t.d41[c];
    be2n[c] += bY2 * t.d21[c] + bY3 * t.d31[c] + bY4 * t.d41[c];
    bd21[c] = bX2 * t.e1n[c] + bY2 * t.e2n[c];
    bd31[c] = bX3 * t.e1n[c] + bY3 * t.e2n[c];
    bd41[c] = bX4 * t.e1n[c] + bY4 * t.e2n[c];
  }
  // ---- CNVEC3 ----
  if (P.ishfram == 2) {
    // e2n = e2p / |e2p| ; e2p = e3n x e1n
    double be2p[3] = {0, 0, 0};
    v_normalize_rev(t.e2n, t.n2, be2n, be2p);
    v_cross_rev(t.e3n, t.e1n, be2p, be3n, be1n);
    // e3n = e3 / |e3| ; e1n = e1p / |e1p|
    double be3[3] = {0, 0, 0}, be1p[3] = {0, 0, 0};
    v_normalize_rev(t.e3n, t.n3, be3n, be3);
    v_normalize_rev(t.e1n, t.n1, be1n, be1p);
    // e1p = q2 e1 + e2 x e3 ; q2 = |e2|^2
    double be1[3], be2[3] = {0, 0, 0};
    for (int c = 0; c < 3; ++c) be1[c] = be1p[c] * t.q2;
    const double bq2 = v_dot(be1p, t.e1);
    v_cross_rev(t.e2, t.e3, be1p, be2, be3);
    for (int c = 0; c < 3; ++c) be2[c] += 2.0 * bq2 * t.e2[c];
    // e3 = e1 x e2
    v_cross_rev(t.e1, t.e2, be3, be1, be2);
    for (int c = 0; c < 3; ++c) {
      bd21[c] += be1[c]; bd34[c] += be1[c];
      bd32[c] += be2[c]; bd41[c] += be2[c];
    }
  } else {
    // e2n = e3n x e1n
    v_cross_rev(t.e3n, t.e1n, be2n, be3n, be1n);
    // e1n = e1p / |e1p|
    double be1p[3] = {0, 0, 0};
    v_normalize_rev(t.e1n, t.n1, be1n, be1p);
    // e1p = e1 + s * (e2 x e3n)
    double be1[3] = {be1p[0], be1p[1], be1p[2]}, be2[3] = {0, 0, 0};
    const double bs = v_dot(be1p, t.c23);
    const double bc23[3] = {be1p[0] * t.s, be1p[1] * t.s, be1p[2] * t.s};
    v_cross_rev(t.e2, t.e3n, bc23, be2, be3n);
    // s = sqrt(q1/q2)
    if (t.s > 0.0) {
      const double bq1 = bs / (2.0 * t.s * t.q2);
      const double bq2 = -bs * t.q1 / (2.0 * t.s * t.q2 * t.q2);
      for (int c = 0; c < 3; ++c) { be1[c] += 2.0 * bq1 * t.e1[c]; be2[c] += 2.0 * bq2 * t.e2[c]; }
    }
    // e3n = e3 / |e3| ; e3 = e1 x e2
    double be3[3] = {0, 0, 0};
    v_normalize_rev(t.e3n, t.n3, be3n, be3);
    v_cross_rev(t.e1, t.e2, be3, be1, be2);
    // e1 = d21 + d34 ; e2 = d32 + d41
    for (int c = 0; c < 3; ++c) {
      bd21[c] += be1[c]; bd34[c] += be1[c];
      bd32[c] += be2[c]; bd41[c] += be2[c];
    }
  }
  for (int c = 0; c < 3; ++c) {
    ib.x[1][c] += bd21[c]; ib.x[0][c] -= bd21[c];
    ib.x[2][c] += bd31[c]; ib.x[0][c] -= bd31[c];
    ib.x[3][c] += bd41[c]; ib.x[0][c] -= bd41[c];
    ib.x[2][c] += bd32[c]; ib.x[1][c] -= bd32[c];
    ib.x[2][c] += bd34[c]; ib.x[3][c] -= bd34[c];
  }
}

}  // namespace orb_adj
