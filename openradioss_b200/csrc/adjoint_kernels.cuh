// adjoint_kernels.cuh -- kernels of the reverse shell cycle (FP64).
//
// One reverse cycle c, given the adjoints of the state after the cycle
// (lamX, lamD, lamV, lamVR per node; lsig, lpla, lthk, lhourg per element):
//
//   adj_node_pre_kernel    reverse of DEPLA, VELOCITY, BCS10 and ACCELE: the
//                          adjoint of the velocities before the cycle, and the
//                          adjoint of each node's assembled force and moment;
//                          accumulates dJ/dMS and dJ/dIN
//   adj_shell_kernel       per element: recompute the element forward from the
//                          stored state, run its reverse (shell_adjoint.cuh),
//                          write the corner adjoints and the element-state
//                          adjoints, accumulate dJ/dA and dJ/dTHKE
//   adj_node_post_kernel   per node: add its corner adjoints in fixed
//                          (element, corner) order to lamX, lamV, lamVR
//
// No float atomics: every sum has a fixed order, so the gradient is bitwise
// reproducible.
#pragma once
#include "ecycle_kernels.cuh"
#include "shell_adjoint.cuh"

namespace orb {

struct AdjGroup {
  orb_adj::ShellParams P;
  int part, has_jca;
  double jc_a;
};

struct AdjNodeArgs {
  const PartDesc* parts;
  const int* tile_part;
  const unsigned char* code;
  const double4* Xn;      // state at the start of the cycle (w = mass)
  const double4* Vn;
  const double4* Vn1;     // velocities after the cycle
  const double4* VRn;     // w = rotational inertia
  const double4* VRn1;
  const PartTime* tnext;  // [part] time at the start of the next cycle: dt2 = DT2, dt12 = DT12
  double4* lamX;
  const double4* lamD;
  double4* lamV;
  double4* lamVR;
  double4* lamF;          // out: adjoint of the assembled nodal force
  double4* lamM;          // out: adjoint of the assembled nodal moment
  double* dms;
  double* din;
  int nnodpad, node_tile;
  const int* skew_of;     // skewed /BCS (code bit 7): frame of the node; may be null
  const double* skews;
};

// reverse of the BCS1V projection: each held direction s is projected out by
// the symmetric I - s s^T, so the transpose applies the same projections in the
// opposite order (for the orthonormal /SKEW frames the two orders agree)
__device__ inline void adj_bcs_skew(int lcod, const double* sk, double b[3]) {
  if (!lcod) return;
  if (lcod == 7) { b[0] = b[1] = b[2] = 0.0; return; }
  auto proj = [&](int r) {
    const double s0 = sk[3 * r], s1 = sk[3 * r + 1], s2 = sk[3 * r + 2];
    const double aa = s0 * b[0] + s1 * b[1] + s2 * b[2];
    b[0] -= s0 * aa; b[1] -= s1 * aa; b[2] -= s2 * aa;
  };
  switch (lcod) {
    case 1: proj(2); break;
    case 2: proj(1); break;
    case 3: proj(1); proj(2); break;
    case 4: proj(0); break;
    case 5: proj(0); proj(2); break;
    case 6: proj(1); proj(0); break;
  }
}

__global__ void __launch_bounds__(128) adj_node_pre_kernel(AdjNodeArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.nnodpad) return;
  const int part = a.tile_part[n / a.node_tile];
  const PartDesc pd = a.parts[part];
  if (n >= pd.node_end) return;
  const PartTime tn = a.tnext[part];
  const double DT2 = tn.dt2, DT12 = tn.dt12;
  const unsigned char code = a.code[n];
  const double4 lx = a.lamX[n], ld = a.lamD[n], lv = a.lamV[n];
  const double4 v0 = a.Vn[n], v1 = a.Vn1[n];
  const double ms = a.Xn[n].w;
  // V(n+1) = V(n) + DT12 * A on free components, 0 on fixed ones; X, D += DT2 * V(n+1)
  double bar[3] = {lv.x + DT2 * (lx.x + ld.x), lv.y + DT2 * (lx.y + ld.y), lv.z + DT2 * (lx.z + ld.z)};
  const double* sk = (code & 128) ? a.skews + 9 * a.skew_of[n] : nullptr;
  const bool fixed[3] = {!sk && (code & 4) != 0, !sk && (code & 2) != 0, !sk && (code & 1) != 0};
  double dv[3] = {v1.x - v0.x, v1.y - v0.y, v1.z - v0.z};
  if (sk) {            // V(n+1) = P V(n) + DT12 P A: the adjoints and A = (V(n+1) - P V(n)) / DT12
    double pv0[3] = {v0.x, v0.y, v0.z};
    bcs1v_skew(code & 7, sk, pv0[0], pv0[1], pv0[2]);
    dv[0] = v1.x - pv0[0]; dv[1] = v1.y - pv0[1]; dv[2] = v1.z - pv0[2];
    adj_bcs_skew(code & 7, sk, bar);
  }
  double lF[3] = {0, 0, 0}, dm = 0.0;
  for (int c = 0; c < 3; ++c) {
    if (fixed[c]) { bar[c] = 0.0; continue; }
    const double lA = DT12 * bar[c];
    if (ms > 0.0) {
      lF[c] = lA / ms;                    // A = F / MS
      dm -= lA * (dv[c] / DT12) / ms;     // dA/dMS = -A / MS
    }
  }
  a.lamV[n] = make_double4(bar[0], bar[1], bar[2], 0.0);
  a.lamF[n] = make_double4(lF[0], lF[1], lF[2], 0.0);
  a.dms[n] += dm;
  if (pd.has_rot) {
    const double4 lr = a.lamVR[n], r0 = a.VRn[n], r1 = a.VRn1[n];
    const double in = r0.w;
    double rb[3] = {lr.x, lr.y, lr.z};
    const bool rfix[3] = {!sk && (code & 32) != 0, !sk && (code & 16) != 0, !sk && (code & 8) != 0};
    double dr[3] = {r1.x - r0.x, r1.y - r0.y, r1.z - r0.z};
    if (sk) {
      double pr0[3] = {r0.x, r0.y, r0.z};
      bcs1v_skew((code >> 3) & 7, sk, pr0[0], pr0[1], pr0[2]);
      dr[0] = r1.x - pr0[0]; dr[1] = r1.y - pr0[1]; dr[2] = r1.z - pr0[2];
      adj_bcs_skew((code >> 3) & 7, sk, rb);
    }
    double lM[3] = {0, 0, 0}, di = 0.0;
    for (int c = 0; c < 3; ++c) {
      if (rfix[c]) { rb[c] = 0.0; continue; }
      const double lA = DT12 * rb[c];
      if (in > 0.0) {
        lM[c] = lA / in;
        di -= lA * (dr[c] / DT12) / in;
      }
    }
    a.lamVR[n] = make_double4(rb[0], rb[1], rb[2], 0.0);
    a.lamM[n] = make_double4(lM[0], lM[1], lM[2], 0.0);
    a.din[n] += di;
  } else {
    a.lamM[n] = make_double4(0, 0, 0, 0);
  }
}

struct AdjShellArgs {
  const AdjGroup* groups;
  const int* egroup;       // group of each internal element, -1 for padding
  const int4* enodes;      // global node of each corner
  const int* degen;
  const double4* Xn;
  const double4* Vn;
  const double4* VRn;
  const double* sig;       // state at the start of the cycle: npt x 5 x nelpad
  const double* pla;       // npt x nelpad
  const double* thk;
  const double* thke;
  const double* hourg;     // 3 x nelpad
  const double* jca;       // may be null
  const PartTime* tcur;    // [part] time at the start of the cycle: dt2 = DT1 of the elements
  const double4* lamF;
  const double4* lamM;
  double* lsig;            // in: adjoint of the state after the cycle; out: before
  double* lpla;
  double* lthk;
  double* lhourg;
  double* dA;
  double* dthke;
  double4* cX;             // per corner (4 x nelpad): adjoint of the corner's x, v, vr
  double4* cV;
  double4* cR;
  const float* zw;
  double w_plastic;
  int nelpad;
};

// Threads per CTA and resident CTAs per SM of the reverse shell kernel (its
// register budget: 65536 / (threads x CTAs) per thread).  64 x 5 (204 registers)
// puts a 40,000-shell plate in one wave of 148 SMs, where 128 x 2 at 255
// registers left a 6 % tail wave: the C5 adjoint 92-93 -> 88.4 ms on B200
// (96 x 3: 88.6 ms); the gradients are bitwise the same.
#ifndef ORB_ADJ_SHELL_THREADS
#define ORB_ADJ_SHELL_THREADS 64
#endif
#ifndef ORB_ADJ_SHELL_CTAS
#define ORB_ADJ_SHELL_CTAS 5
#endif
constexpr int ADJ_SHELL_THREADS = ORB_ADJ_SHELL_THREADS;

template <int NP>
__global__ void __launch_bounds__(ADJ_SHELL_THREADS, ORB_ADJ_SHELL_CTAS) adj_shell_kernel(AdjShellArgs a) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.nelpad) return;
  const int gi = a.egroup[e];
  if (gi < 0) return;
  const AdjGroup G = a.groups[gi];
  orb_adj::ShellParams P = G.P;
  P.degen = a.degen[e];
  const int npt = P.npt < NP ? P.npt : NP;
  const int nelpad = a.nelpad;
  const int4 nd = a.enodes[e];
  const int node[4] = {nd.x, nd.y, nd.z, nd.w};
  orb_adj::ShellIn<NP> in;
  orb_adj::ShellOut<NP> ob;
  for (int k = 0; k < 4; ++k) {
    const double4 x = a.Xn[node[k]], v = a.Vn[node[k]], r = a.VRn[node[k]];
    in.x[k][0] = x.x; in.x[k][1] = x.y; in.x[k][2] = x.z;
    in.v[k][0] = v.x; in.v[k][1] = v.y; in.v[k][2] = v.z;
    in.vr[k][0] = r.x; in.vr[k][1] = r.y; in.vr[k][2] = r.z;
    const double4 f = a.lamF[node[k]], m = a.lamM[node[k]];
    ob.f[k][0] = f.x; ob.f[k][1] = f.y; ob.f[k][2] = f.z;
    ob.m[k][0] = m.x; ob.m[k][1] = m.y; ob.m[k][2] = m.z;
  }
  for (int ip = 0; ip < NP; ++ip) {
    for (int c = 0; c < 5; ++c) {
      in.sig[ip][c] = ip < npt ? a.sig[(ip * 5 + c) * nelpad + e] : 0.0;
      ob.sig[ip][c] = ip < npt ? a.lsig[(ip * 5 + c) * nelpad + e] : 0.0;
    }
    in.pla[ip] = ip < npt ? a.pla[ip * nelpad + e] : 0.0;
    ob.pla[ip] = ip < npt ? a.lpla[ip * nelpad + e] : 0.0;
  }
  in.thk = a.thk[e];
  in.thke = a.thke[e];
  for (int q = 0; q < 3; ++q) { in.hourg[q] = a.hourg[q * nelpad + e]; ob.hourg[q] = a.lhourg[q * nelpad + e]; }
  in.ca = G.has_jca ? a.jca[e] : G.jc_a;
  in.dt1 = a.tcur[G.part].dt2;
  ob.thk = a.lthk[e];
  ob.wpla = a.w_plastic;
  orb_adj::ShellTape<NP> t;
  orb_adj::ShellOut<NP> out;
  orb_adj::shell_forward<NP>(P, a.zw, in, out, t);
  orb_adj::ShellIn<NP> ib;
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) { ib.x[k][c] = 0.0; ib.v[k][c] = 0.0; ib.vr[k][c] = 0.0; }
  for (int ip = 0; ip < NP; ++ip) {
    for (int c = 0; c < 5; ++c) ib.sig[ip][c] = 0.0;
    ib.pla[ip] = 0.0;
  }
  ib.thk = ib.thke = ib.ca = ib.dt1 = 0.0;
  ib.hourg[0] = ib.hourg[1] = ib.hourg[2] = 0.0;
  orb_adj::shell_reverse<NP>(P, a.zw, in, t, ob, ib);
  for (int ip = 0; ip < npt; ++ip) {
    for (int c = 0; c < 5; ++c) a.lsig[(ip * 5 + c) * nelpad + e] = ib.sig[ip][c];
    a.lpla[ip * nelpad + e] = ib.pla[ip];
  }
  a.lthk[e] = ib.thk;
  for (int q = 0; q < 3; ++q) a.lhourg[q * nelpad + e] = ib.hourg[q];
  a.dA[e] += ib.ca;
  a.dthke[e] += ib.thke;
  for (int k = 0; k < 4; ++k) {
    a.cX[4 * e + k] = make_double4(ib.x[k][0], ib.x[k][1], ib.x[k][2], 0.0);
    a.cV[4 * e + k] = make_double4(ib.v[k][0], ib.v[k][1], ib.v[k][2], 0.0);
    a.cR[4 * e + k] = make_double4(ib.vr[k][0], ib.vr[k][1], ib.vr[k][2], 0.0);
  }
}

struct AdjPostArgs {
  const int* ofs;          // nnodpad + 1: corner entries of each node
  const int* ent;          // corner ids (4 * element + corner), ascending
  const double4* cX;
  const double4* cV;
  const double4* cR;
  double4* lamX;
  double4* lamV;
  double4* lamVR;
  int nnodpad;
};

__global__ void __launch_bounds__(128) adj_node_post_kernel(AdjPostArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.nnodpad) return;
  const int k0 = a.ofs[n], k1 = a.ofs[n + 1];
  if (k1 == k0) return;
  double4 x = a.lamX[n], v = a.lamV[n], r = a.lamVR[n];
  for (int k = k0; k < k1; ++k) {
    const int j = a.ent[k];
    const double4 cx = a.cX[j], cv = a.cV[j], cr = a.cR[j];
    x.x += cx.x; x.y += cx.y; x.z += cx.z;
    v.x += cv.x; v.y += cv.y; v.z += cv.z;
    r.x += cr.x; r.y += cr.y; r.z += cr.z;
  }
  a.lamX[n] = x;
  a.lamV[n] = v;
  a.lamVR[n] = r;
}

}  // namespace orb
