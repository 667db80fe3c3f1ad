// persistent_kernel.cuh -- the whole explicit cycle of a shell mesh in one launch.
//
// For a mesh whose element and nodal state fit on the chip (one part of BT
// shells, C2-sized), shell_persistent_kernel runs all the cycles of a step in a
// single cooperative launch of one CTA per SM:
//
//   per cycle   element phase   every CTA computes its patches (the same patches,
//                               element arithmetic and incidence-list sums as
//                               shell_patch_kernel) from nodal state it keeps in
//                               shared memory and element state it keeps in
//                               registers, writes the patch partial sums to the
//                               node-major slot skyline and min-reduces the time step
//               grid barrier    (one per cycle)
//               node phase      every CTA updates all the nodes its patches touch
//                               (ASSPAR4 over the skyline slots in patch order, the
//                               dt logic, ACCELE, BCS10, VELOCITY, DEPLA: the same
//                               node_update as the node pass), so a node shared by
//                               several CTAs is updated identically by each of them
//
// Only the skyline slots and the time-step reduction cross between SMs (through
// L2).  The slots are double-buffered by cycle parity and the reduction is
// triple-buffered, so one barrier per cycle orders every reuse.  The result is
// bit for bit the result of the patch and node kernels: the same operations in
// the same order.  After the last cycle each node's owner (the lowest CTA that
// holds it) writes it back, the element state is written back, and the kinetic
// energy is summed per node tile exactly as the node pass sums it.
//
// The barrier is a monotonic arrival counter polled with a time limit: past the
// limit a CTA sets an abort flag and the OR_E_TIMEOUT error word, and every CTA
// leaves at its next barrier, so the launch always ends.
#pragma once
#include "ecycle_kernels.cuh"

namespace orb {

// host-built layout of the persistent launch (one part, shell groups only)
struct PersistArgs {
  const int* node_ofs;        // G + 1: CTA c holds nodes node_ofs[c] .. node_ofs[c+1]-1 of the lists below
  const int* node_glob;       // padded global node number of each held node, ascending within a CTA
  const unsigned char* owner; // 1 where the CTA is the lowest that holds the node
  const uint2* pconn;         // per padded shell element: 4 x uint16 CTA-local node indices
  void* fslot2;               // second slot buffers (odd cycles); the handle's fslot / mslot serve even ones
  void* mslot2;
  PartAcc* acc3;              // triple-buffered time-step reduction
  double* ek_node;            // last cycle's kinetic energy of every node (owners write)
  double* ekr_node;
  unsigned* sync;             // [0] arrival counter, [1] abort flag
  int patches_per_cta;        // P
  int ncmax;                  // node capacity of a CTA (stride of the shared planes)
  int ntiles_node;            // node tiles of NODE tile size 128 (kinetic energy partials)
  int stall_cta;              // test hook (OR_ECYCLE_TEST_STALL_CTA): this CTA does not arrive at the
                              // first cycle's barrier, so the others' bounded waits run out; -1 off
};

// L2-coherent loads and stores (bypassing L1) of the data other SMs write during
// the launch: the slot skyline and the reduction
__device__ __forceinline__ float4 ld_cg(const float4* p) { return __ldcg(p); }
__device__ __forceinline__ double4 ld_cg(const double4* p) {
  const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st_cg(float4* p, float4 v) { __stcg(p, v); }
__device__ __forceinline__ void st_cg(double4* p, double4 v) {
  __stcg(reinterpret_cast<double2*>(p), make_double2(v.x, v.y));
  __stcg(reinterpret_cast<double2*>(p) + 1, make_double2(v.z, v.w));
}

// one grid-wide barrier: arrive, then poll the counter until every CTA arrived at
// this barrier; true when the launch must end (a CTA gave up waiting)
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ bool grid_barrier(unsigned* sync, unsigned target, ErrorWord* err, int* s_abort,
                                             bool arrive = true) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();                          // release: this CTA's slot writes and reductions
    if (arrive) atomicAdd(&sync[0], 1u);
    const long long t0 = clock64();
    int ab = 0;
    for (;;) {
      const unsigned v = ld_acquire(&sync[0]);  // acquire: every CTA's writes before its arrival
      if (v >= target) break;
      if (__ldcg(&sync[1])) { ab = 1; break; }
      if (clock64() - t0 > (1ll << 31)) {           // about a second at the SM clock
        atomicExch(&sync[1], 1u);
        raise_error(err, 7, (int)blockIdx.x);
        ab = 1;
        break;
      }
      __nanosleep(32);
    }
    if (ab) __threadfence();
    *s_abort = ab;
  }
  __syncthreads();
  return *s_abort != 0;
}

// pairs of reals for the corner-force planes of the persistent kernel
template <class R> struct Vec2;
template <> struct Vec2<float> { typedef float2 T; };
template <> struct Vec2<double> { typedef double2 T; };
__device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }

// the dt-key / dt-bits min and the two energy sums of a group of TILE threads
// (threads g*TILE .. g*TILE+TILE-1), with the operation order of block_reduce
template <int TILE>
__device__ inline void group_reduce(unsigned long long& key, unsigned long long& bits, double& s0, double& s1,
                                    unsigned long long* skey, unsigned long long* sbits, double* ss0, double* ss1) {
  const int lt = threadIdx.x % TILE;
  const int lane = lt & 31, warp = lt >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
    unsigned long long b2 = __shfl_xor_sync(0xffffffffu, bits, o);
    key = k2 < key ? k2 : key;
    bits = b2 < bits ? b2 : bits;
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  if (lane == 0) { skey[warp] = key; sbits[warp] = bits; ss0[warp] = s0; ss1[warp] = s1; }
  __syncthreads();
  if (warp == 0) {
    constexpr int NW = TILE / 32;
    key = lane < NW ? skey[lane] : ~0ull;
    bits = lane < NW ? sbits[lane] : ~0ull;
    s0 = lane < NW ? ss0[lane] : 0.0;
    s1 = lane < NW ? ss1[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
      unsigned long long b2 = __shfl_xor_sync(0xffffffffu, bits, o);
      key = k2 < key ? k2 : key;
      bits = b2 < bits ? b2 : bits;
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
  }
}

// Threads per CTA: at least P patches x TILE elements (one per element), raised to
// cover the CTA's held nodes (one per node in the node phase) and at most
// PERSIST_THREADS; one CTA per SM (the register budget of the shell element at that
// many threads).  Threads beyond the P patches work in the node phase only.
constexpr int PERSIST_THREADS = 384;
// reduction scratch is laid out for every TILE group of PERSIST_THREADS threads
__host__ __device__ constexpr int persist_groups(int tile) { return (PERSIST_THREADS + tile - 1) / tile; }

template <class R>
__host__ __device__ inline size_t persist_smem(int ncmax, int tile, int P, int inc_stride, int nlmax) {
  // node planes: x y z dx dy dz (FP64), vx vy vz rx ry rz ms in (R), global index
  // (int), owner and code (bytes); per patch: 24 corner planes of TILE (R), the
  // incidence lists (uint16), reduction scratch, the slot of each patch node (int);
  // per held node its slot range (int2)
  const size_t nodes = (size_t)ncmax * (6 * sizeof(double) + 8 * sizeof(R) + sizeof(int) + 2);
  const size_t nodes_al = (nodes + 15) / 16 * 16;
  const size_t corners = (size_t)P * 24 * tile * sizeof(R);
  const size_t inc = ((size_t)P * inc_stride * 2 + 15) / 16 * 16;
  const size_t red = (size_t)persist_groups(tile) * (tile / 32) * 32;
  const size_t slots = ((size_t)P * nlmax * sizeof(int) + 15) / 16 * 16;
  const size_t ranges = (size_t)ncmax * sizeof(int2);
  return nodes_al + corners + inc + red + slots + ranges;
}

template <class R, int TILE, int NPT>
__global__ void __launch_bounds__(PERSIST_THREADS, 1)
shell_persistent_kernel(ShellArgs<R> a, NodeArgs<R> na, PersistArgs pa, int ncycles, int parity0,
                        const float* __restrict__ zw) {
  typedef typename Vec4<R>::T R4;
  constexpr bool KEEP = NPT > 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_abort;
  __shared__ double s_e0[PERSIST_THREADS / 32], s_e1[PERSIST_THREADS / 32];
  __shared__ unsigned long long s_dt[2];        // the CTA's dt key and dt bits minimum of a cycle
  const int tid = threadIdx.x;
  const int cta = blockIdx.x, G = gridDim.x;
  const int P = pa.patches_per_cta, NC = pa.ncmax;
  const int sub = tid / TILE, lt = tid % TILE;
  // ---- shared layout ----
  double* sx = reinterpret_cast<double*>(smem_raw);
  double* sy = sx + NC;
  double* sz = sy + NC;
  double* sdx = sz + NC;
  double* sdy = sdx + NC;
  double* sdz = sdy + NC;
  R* sv = reinterpret_cast<R*>(sdz + NC);      // vx vy vz rx ry rz: 6 planes of NC
  R* sms = sv + 6 * NC;
  R* sin_ = sms + NC;
  int* sglob = reinterpret_cast<int*>(sin_ + NC);
  unsigned char* sown = reinterpret_cast<unsigned char*>(sglob + NC);
  unsigned char* scode = sown + NC;
  const size_t nodes = (size_t)NC * (6 * sizeof(double) + 8 * sizeof(R) + sizeof(int) + 2);
  unsigned char* after_nodes = smem_raw + (nodes + 15) / 16 * 16;
  R* sc_all = reinterpret_cast<R*>(after_nodes);                  // P x 24 x TILE
  unsigned short* sinc_all = reinterpret_cast<unsigned short*>(sc_all + (size_t)P * 24 * TILE);
  unsigned char* red_base = reinterpret_cast<unsigned char*>(sinc_all) + ((size_t)P * a.inc_stride * 2 + 15) / 16 * 16;
  constexpr int NW = TILE / 32;
  unsigned long long* s_key = reinterpret_cast<unsigned long long*>(red_base) + sub * 4 * NW;
  unsigned long long* s_bits = s_key + NW;
  double* s_s0 = reinterpret_cast<double*>(s_bits + NW);
  double* s_s1 = s_s0 + NW;
  R* sc = sc_all + (size_t)sub * 24 * TILE;
  unsigned short* sinc = sinc_all + (size_t)sub * a.inc_stride;
  // slot numbers of the patch nodes and slot ranges of the held nodes, read once
  // here instead of from global memory in every cycle
  int* sslot_all = reinterpret_cast<int*>(red_base + (size_t)persist_groups(TILE) * NW * 32);
  int* sslot = sslot_all + (size_t)sub * a.nlmax;
  int2* srange = reinterpret_cast<int2*>(reinterpret_cast<unsigned char*>(sslot_all) +
                                         ((size_t)P * a.nlmax * sizeof(int) + 15) / 16 * 16);

  // ---- this CTA's patch and element ----
  const int p = cta * P + sub;
  const bool has_patch = sub < P && p < a.npatch;
  const int e = (has_patch ? p : 0) * TILE + lt;
  PatchInfo pi{};
  if (has_patch) pi = a.patch[p];
  const bool active = has_patch && lt < pi.nel;
  const int NLM = a.nlmax;
  // ---- stage the held nodes, the incidence lists, the element state ----
  const int n0 = pa.node_ofs[cta], nn = pa.node_ofs[cta + 1] - n0;
  for (int i = tid; i < nn; i += blockDim.x) {
    const int g = pa.node_glob[n0 + i];
    const double4 xx = na.X[g];
    const R4 vv = na.V[g];
    const R4 rr = na.VR[g];
    sx[i] = xx.x; sy[i] = xx.y; sz[i] = xx.z;
    sdx[i] = na.DX[g]; sdy[i] = na.DY[g]; sdz[i] = na.DZ[g];
    sv[0 * NC + i] = vv.x; sv[1 * NC + i] = vv.y; sv[2 * NC + i] = vv.z;
    sv[3 * NC + i] = rr.x; sv[4 * NC + i] = rr.y; sv[5 * NC + i] = rr.z;
    sms[i] = R(xx.w);
    sin_[i] = rr.w;
    sglob[i] = g;
    sown[i] = pa.owner[n0 + i];
    scode[i] = na.code[g];
    srange[i] = make_int2(na.adsky[g], na.adsky[g + 1]);
  }
  if (has_patch) {
    const unsigned* src = reinterpret_cast<const unsigned*>(a.inc + (size_t)p * a.inc_stride);
    unsigned* dst = reinterpret_cast<unsigned*>(sinc);
    for (int i = lt; i < a.inc_stride / 2; i += TILE) dst[i] = src[i];
    for (int j = lt; j < a.patch[p].nloc; j += TILE) sslot[j] = a.patch_slots[p * a.nlmax + j];
  }
  ShellState<R, NPT> st;
  if (KEEP) shell_load_state<R, NPT>(a, e, st);
  int lc[4] = {0, 0, 0, 0};
  {
    const uint2 w = pa.pconn[e];
    lc[0] = w.x & 0xffffu; lc[1] = w.x >> 16; lc[2] = w.y & 0xffffu; lc[3] = w.y >> 16;
  }
  const ShellGroupDesc gd = a.groups[has_patch ? pi.group : 0];
  const int nl = has_patch ? pi.nloc : 0;
  // Energies: each thread adds its element's hourglass energy and plastic work over
  // the launch's cycles; the patch sums them once at the end onto its cumulative
  // partials (the phase kernels sum per cycle, so the two agree to FP64 rounding).
  double cum_ehou_t = 0.0, cum_wpla_t = 0.0;
  if (tid == 0) { s_dt[0] = ~0ull; s_dt[1] = ~0ull; }
  PartTime t = na.time[parity0];
  R4* fs[2] = {a.fslot, reinterpret_cast<R4*>(pa.fslot2)};
  R4* ms_[2] = {a.mslot, reinterpret_cast<R4*>(pa.mslot2)};
  __syncthreads();

  for (int c = 0; c < ncycles; ++c) {
    R4* fslot = fs[c & 1];
    R4* mslot = ms_[c & 1];
    // ---------------- element phase ----------------
    const R DT1 = R(t.dt2);
    R Fg[3][4], Mg[3][4];
    unsigned long long mykey = ~0ull, mybits = ~0ull;
    double my_ehou = 0.0, my_wpla = 0.0;
    if (active) {
      if (!KEEP) shell_load_state<R, NPT>(a, e, st);
      shell_element<R, NPT, KEEP>(a, e, gd, DT1, zw, sx, sy, sz, sv, NC, lc, st, Fg, Mg, mykey, mybits, my_ehou,
                                  my_wpla);
      // corner forces and moments as three planes of pairs (fx fy | fz mx | my mz),
      // corner k of element lt at k * TILE + lt
      typename Vec2<R>::T* sc2 = reinterpret_cast<typename Vec2<R>::T*>(sc);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        sc2[(0 * 4 + k) * TILE + lt] = mk2(Fg[0][k], Fg[1][k]);
        sc2[(1 * 4 + k) * TILE + lt] = mk2(Fg[2][k], Mg[0][k]);
        sc2[(2 * 4 + k) * TILE + lt] = mk2(Mg[1][k], Mg[2][k]);
      }
      cum_ehou_t += my_ehou;
      cum_wpla_t += my_wpla;
    }
    {   // the CTA's dt minimum: per warp in registers, then one shared atomic per warp
      const unsigned long long wk = warp_min_u64(mykey), wb = warp_min_u64(mybits);
      if ((tid & 31) == 0) { atomicMin(&s_dt[0], wk); atomicMin(&s_dt[1], wb); }
    }
    __syncthreads();
    if (tid == 0) {      // to the grid's reduction at once, ahead of the patch sums
      PartAcc* acc = &pa.acc3[c % 3];
      atomicMin(&acc->dtkey, s_dt[0]);
      atomicMin(&acc->dtbits, s_dt[1]);
      s_dt[0] = ~0ull; s_dt[1] = ~0ull;        // no warp touches them again before the grid barrier
    }
    for (int j = lt; j < nl; j += TILE) {
      R f0 = R(0), f1 = R(0), f2 = R(0), m0 = R(0), m1 = R(0), m2 = R(0);
      const int i1 = sinc[j + 1];
      const typename Vec2<R>::T* sc2 = reinterpret_cast<const typename Vec2<R>::T*>(sc);
#pragma unroll 4
      for (int i = sinc[j]; i < i1; ++i) {
        const int o = sinc[NLM + 1 + i];   // corner k of element t: k * TILE + t
        const typename Vec2<R>::T p0 = sc2[o], p1 = sc2[4 * TILE + o], p2 = sc2[8 * TILE + o];
        f0 += p0.x; f1 += p0.y; f2 += p1.x;
        m0 += p1.y; m1 += p2.x; m2 += p2.y;
      }
      const int s = sslot[j];
      st_cg(&fslot[s], mk4(f0, f1, f2, R(0)));
      st_cg(&mslot[s], mk4(m0, m1, m2, R(0)));
    }
    if (grid_barrier(pa.sync, (unsigned)(c + 1) * (unsigned)G, a.err, &s_abort, !(c == 0 && cta == pa.stall_cta)))
      return;
    // ---------------- node phase ----------------
    // A thread's nodes are i0 = tid + 2 j blockDim.x and i0 + blockDim.x.  The first
    // two slots of both are loaded before either is summed, and for the first pair
    // before the cycle's dt reduction is read, so that all these L2 reads are in
    // flight together.
    R4 F0[2], F1[2], M0[2], M1[2];
    int2 rg[2];
    auto prefetch = [&](int i0) {
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int i = i0 + u * blockDim.x;
        rg[u] = i < nn ? srange[i] : make_int2(0, 0);
        F0[u] = F1[u] = M0[u] = M1[u] = mk4(R(0), R(0), R(0), R(0));
        if (rg[u].y > rg[u].x) { F0[u] = ld_cg(&fslot[rg[u].x]); M0[u] = ld_cg(&mslot[rg[u].x]); }
        if (rg[u].y > rg[u].x + 1) { F1[u] = ld_cg(&fslot[rg[u].x + 1]); M1[u] = ld_cg(&mslot[rg[u].x + 1]); }
      }
    };
    prefetch(tid);
    PartAcc ac;
    ac.dtkey = __ldcg(&pa.acc3[c % 3].dtkey);
    ac.dtbits = __ldcg(&pa.acc3[c % 3].dtbits);
    int ityp, nelt;
    double DT2;
    cycle_dt(ac, t, na.growth, na.dtmx, na.split, DT2, ityp, nelt);
    const double DTc1 = t.dt2;
    const double DT12 = 0.5 * (DTc1 + DT2);
    const bool last = c == ncycles - 1;
    for (int i0 = tid; i0 < nn; i0 += 2 * blockDim.x) {
    if (i0 != tid) prefetch(i0);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i >= nn) break;
      const int g = sglob[i];
      const int k0 = rg[u].x, k1 = rg[u].y;
      R ax = R(0), ay = R(0), az = R(0), rx = R(0), ry = R(0), rz = R(0);
      if (k1 > k0) {
        ax = F0[u].x; ay = F0[u].y; az = F0[u].z;
        rx = M0[u].x; ry = M0[u].y; rz = M0[u].z;
      }
      if (k1 > k0 + 1) {
        ax += F1[u].x; ay += F1[u].y; az += F1[u].z;
        rx += M1[u].x; ry += M1[u].y; rz += M1[u].z;
      }
      for (int k = k0 + 2; k < k1; ++k) {
        const R4 f = ld_cg(&fslot[k]);
        ax += f.x; ay += f.y; az += f.z;
        const R4 m = ld_cg(&mslot[k]);
        rx += m.x; ry += m.y; rz += m.z;
      }
      double px = sx[i], py = sy[i], pz = sz[i], qx = sdx[i], qy = sdy[i], qz = sdz[i];
      R4 v = mk4(sv[0 * NC + i], sv[1 * NC + i], sv[2 * NC + i], R(0));
      R4 w = mk4(sv[3 * NC + i], sv[4 * NC + i], sv[5 * NC + i], sin_[i]);
      double ek = 0.0, ekr = 0.0;
      node_update<R>(na, g, scode[i], true, ax, ay, az, rx, ry, rz, sms[i], DTc1, DT2, DT12, px, py, pz, qx, qy, qz,
                     v, w, ek, ekr, last);        // only the launch's last cycle reports kinetic energy
      sx[i] = px; sy[i] = py; sz[i] = pz; sdx[i] = qx; sdy[i] = qy; sdz[i] = qz;
      sv[0 * NC + i] = v.x; sv[1 * NC + i] = v.y; sv[2 * NC + i] = v.z;
      sv[3 * NC + i] = w.x; sv[4 * NC + i] = w.y; sv[5 * NC + i] = w.z;
      if (last && sown[i]) { pa.ek_node[g] = ek; pa.ekr_node[g] = ekr; }
    }
    }
    if (cta == 0 && tid == 0) {            // reuse in two cycles: everyone has read it
      PartAcc r; r.dtkey = ~0ull; r.dtbits = ~0ull;
      pa.acc3[(c + 2) % 3] = r;
    }
    t.tt = t.tt + DT2; t.dt2 = DT2; t.dt2old = DT2; t.dt1 = DTc1; t.dt12 = DT12;
    t.ncycle = t.ncycle + 1; t.ityptst = ityp; t.neltst = nelt; t.pad = 0;
    __syncthreads();
  }

  // ---- write back: held nodes by their owner, element state, energies, time ----
  for (int i = tid; i < nn; i += blockDim.x) {
    if (!sown[i]) continue;
    const int g = sglob[i];
    na.X[g] = make_double4(sx[i], sy[i], sz[i], na.X[g].w);
    na.DX[g] = sdx[i]; na.DY[g] = sdy[i]; na.DZ[g] = sdz[i];
    na.V[g] = mk4(sv[0 * NC + i], sv[1 * NC + i], sv[2 * NC + i], R(0));
    na.VR[g] = mk4(sv[3 * NC + i], sv[4 * NC + i], sv[5 * NC + i], sin_[i]);
  }
  if constexpr (KEEP) {
    if (has_patch) shell_store_state<R, NPT>(a, e, st);
  }
  {
    unsigned long long k0 = ~0ull, k1 = ~0ull;
    group_reduce<TILE>(k0, k1, cum_ehou_t, cum_wpla_t, s_key, s_bits, s_s0, s_s1);
    if (has_patch && lt == 0) {
      a.blk_ehour[p] = a.blk_ehour[p] + cum_ehou_t;
      a.blk_wpla[p] = a.blk_wpla[p] + cum_wpla_t;
    }
  }
  if (cta == 0 && tid == 0) {
    const int fin = (parity0 + ncycles) & 1;
    na.time[fin] = t;
    PartAcc r; r.dtkey = ~0ull; r.dtbits = ~0ull;
    a.acc[fin] = r;
  }
  // kinetic energy per node tile of 128, summed as the node pass sums it
  if (grid_barrier(pa.sync, (unsigned)(ncycles + 1) * (unsigned)G, a.err, &s_abort)) return;
  for (int tile = cta; tile < pa.ntiles_node; tile += G) {
    double ek = 0.0, ekr = 0.0;
    if (tid < 128) {
      ek = __ldcg(&pa.ek_node[tile * 128 + tid]);
      ekr = __ldcg(&pa.ekr_node[tile * 128 + tid]);
    }
    const int lane = tid & 31, warp = tid >> 5;
    if (tid < 128) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ek += __shfl_xor_sync(0xffffffffu, ek, o);
        ekr += __shfl_xor_sync(0xffffffffu, ekr, o);
      }
      if (lane == 0) { s_e0[warp] = ek; s_e1[warp] = ekr; }
    }
    __syncthreads();
    if (tid == 0) {
      double s0 = 0.0, s1 = 0.0;
      for (int w = 0; w < 4; ++w) { s0 += s_e0[w]; s1 += s_e1[w]; }
      na.blk_ekin[tile] = s0;
      na.blk_ekinr[tile] = s1;
    }
    __syncthreads();
  }
}

}  // namespace orb
