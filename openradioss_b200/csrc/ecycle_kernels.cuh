// ecycle_kernels.cuh -- sm_100a kernels of the explicit element cycle.
//
// Three kernels per cycle:
//   hex_patch_kernel    SFORC3 chain for 8-node 1-point hexas (+ LAW1/LAW2)
//   shell_patch_kernel  CFORC3 chain for BT shells (+ LAW1/LAW2 plane stress)
//   node_kernel         ASSPAR4 + dt logic + ACCELE + BCS10 + VELOCITY + DEPLA
//
// Elements are grouped into patches of at most TILE elements (one CTA each).
// A patch lists its unique nodes; the CTA stages their coordinates and
// velocities in shared memory, each thread computes one element, and the
// corner forces are reduced into shared-memory node accumulators colour by
// colour (no two elements of a colour share a node), so the sum order is fixed
// and no float atomics are used.  Each (patch, node) partial sum is written to
// one slot of a node-major skyline; the node kernel adds a node's slots in
// ascending patch order (the Parith/ON idea of asspar4.F:160-175 applied to
// patch partials instead of element corners).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace orb {

constexpr double EM15 = 1e-15, EM20 = 1e-20, EM30 = 1e-30;
constexpr int MAX_COLORS = 32;
constexpr int COLOR_SHIFT = 11;            // local node index < 2048, colour in bits 11..15
constexpr unsigned LOCAL_MASK = (1u << COLOR_SHIFT) - 1u;

template <class R> struct Vec4;
template <> struct Vec4<float> { typedef float4 T; };
template <> struct Vec4<double> { typedef double4 T; };

__host__ __device__ inline float4 mk4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
__host__ __device__ inline double4 mk4(double a, double b, double c, double d) { return make_double4(a, b, c, d); }

// ---------------------------------------------------------------------------
// descriptors (built on the host at finalize, read-only on the device)
// ---------------------------------------------------------------------------
struct PatchInfo {
  int group;      // group index (hex or shell table)
  int nel;        // elements in this patch (<= TILE)
  int node_ofs;   // offset into patch_nodes / patch_slots
  int nloc;       // unique local nodes
  int ncolor;     // colours used
  int elem0;      // first element (padded internal index) of this patch
  int part;       // part of the patch's group (time state, dt reduction target)
  int pad1;
};

struct HexGroupDesc {
  int part, law, nel, jcvt;       // jcvt: 1 = convected frame (Iframe 2)
  double rho0, shear, bulk, jc_a, jc_b, jc_n, epsmax, sigmax;
  double qa, qb, qh, dtfac, dtmin;
  double pad;                     // 128 bytes: the hexa kernel stages it by bulk copy
};
static_assert(sizeof(HexGroupDesc) % 16 == 0, "HexGroupDesc is bulk-copied");

struct ShellGroupDesc {
  int part, law, nel, npt;
  int ithk, has_jca, ishfram, ipla;   // ipla: M2CPLR return (0 radial, 1 Newton, 2 projection)
  int ihbe, pad;                      // engine IHBE (IPARG(23)): 1, 0, 2 or 4
  double rho0, young, nu, shear, a11, a12, ssp, jc_a, jc_b, jc_n, sigmax;
  double hm, hf, hr, shf, pressure, dtfac, dtmin;
  double dn;                          // GEO(17): one-point V-shape hourglass coefficient
};

struct PartDesc {
  int node_start, node_end;  // padded global node range
  int tile_start, has_rot;
};

// time state of a part at the START of a cycle (double-buffered by parity)
struct PartTime {
  double tt, dt2, dt2old, dt1, dt12;
  int ncycle, ityptst, neltst, pad;
};

// per-part reduction targets of one cycle
struct PartAcc {
  unsigned long long dtkey;   // (float(dt) bits << 32) | (type<<31 | element), min
  unsigned long long dtbits;  // exact dt bits (double), min
};

// one load of FORCE (force.F90): a /CLOAD node (type 0) or a /PLOAD segment (type 1)
struct LoadDesc {
  int type, part, func, dir;      // dir: 1..6 for a /CLOAD; 3 or 4 corners for a /PLOAD
  int skew, pad;                  // /CLOAD skew frame, -1 = global axes
  int node[4], slot[4];           // padded global node numbers and their assembly slots
  double fcx, fcy;                // 1 / Ascale_x, Fscale_y
};
struct FuncDesc {
  int first, count;               // points in the function tables
};

// rigid velocity link (/VEL/TRA, /VEL/ROT; rlink1.F): its nodes and directions
struct LinkDesc {
  int first, count;     // node range in link_nodes (global padded node numbers)
  int ic, icr;          // translation / rotation directions, 4=x 2=y 1=z, 0 = off
};
// mean accelerations of one link in the current cycle (link_kernel)
struct LinkMean {
  double a[3], ar[3];
  int ic, icr;          // directions applied: 0 where the link's mass (inertia) is zero
};

struct ErrorWord {
  int code;
  int index;
};

template <class R>
struct HexArgs {
  const PatchInfo* patch;
  const HexGroupDesc* groups;
  const int* patch_nodes;     // nlmax per patch; padding repeats a node of the patch
  const int* patch_slots;     // nlmax per patch; padding -1
  const uint4* conn;          // 8 x uint16 local corners per element (colour in corner 0)
  const unsigned short* inc;  // per patch (stride inc_stride): nlmax+1 offsets, then the
                              // patch nodes' incident corners (t, k) in ascending order, stored as k*TILE+t
  const int* elem_id;         // element number within its part (for NELTS)
  const double4* X;           // x, y, z, nodal mass
  const typename Vec4<R>::T* V;
  R* sig;                     // 6 x nelpad component-major
  R* eint; R* rho; R* qvis; R* pla; R* epsd;
  const R* vol0; const double* vol0dp;
  typename Vec4<R>::T* fslot;
  const PartTime* time;       // [parity][part]
  PartAcc* acc;               // [parity][part]
  double* blk_ehour;          // per patch cumulative hourglass energy
  double* blk_wpla;           // per patch cumulative plastic work
  ErrorWord* err;
  int nelpad, nparts, npatch;
  int nlmax;                  // stride of patch_nodes / patch_slots (padded per patch)
  int inc_stride;
};

template <class R>
struct ShellArgs {
  const PatchInfo* patch;
  const ShellGroupDesc* groups;
  const int* patch_nodes;     // nlmax per patch; padding repeats a node of the patch
  const int* patch_slots;     // nlmax per patch; padding -1
  const uint2* conn;          // 4 x uint16 local corners per element (colour in corner 0)
  const unsigned short* inc;  // per patch (stride inc_stride): nlmax+1 offsets, then the
                              // patch nodes' incident corners (t, k) in ascending order, stored as k*TILE+t
  const int* elem_id;
  const int* degen;           // 1 if IXC(4)==IXC(5) (triangle stored as quad)
  const double4* X;
  const typename Vec4<R>::T* V;
  const typename Vec4<R>::T* VR;
  R* sig;                     // npt x 5 x nelpad
  R* pla;                     // npt x nelpad
  R* thk; const R* thke; R* hourg; R* eint; const R* jca;
  typename Vec4<R>::T* fslot;
  typename Vec4<R>::T* mslot;
  const PartTime* time;
  PartAcc* acc;
  double* blk_ehour;
  double* blk_wpla;
  ErrorWord* err;
  int nelpad, nparts, npatch, maxnpt;
  int nlmax;                  // stride of patch_nodes / patch_slots (padded per patch)
  int inc_stride;
};

template <class R>
struct NodeArgs {
  const PartDesc* parts;
  const int* tile_part;
  const int* adsky;           // nnodpad + 1
  const typename Vec4<R>::T* fslot;
  const typename Vec4<R>::T* mslot;   // may be null
  double4* X;
  double* DX; double* DY; double* DZ;
  typename Vec4<R>::T* V;
  typename Vec4<R>::T* VR;    // w = rotational inertia; may be null
  const unsigned char* code;  // bits 0-2 ICODT, 3-5 ICODR
  PartTime* time;
  PartAcc* acc;
  double* blk_ekin;           // per node tile, overwritten each cycle
  double* blk_ekinr;
  ErrorWord* err;
  double growth, dtmx;
  int ntiles, nparts, split;
  // Domain decomposition (one part split over ranks); halo_slot is null otherwise.
  // A node shared with other ranks takes its force and moment as the sum of every
  // rank's partial sum, rank by rank, from the gathered exchange buffers; the
  // time step is the minimum of every rank's reduction.
  const int* halo_slot;            // per node: its slot in the exchange buffers, or -1
  const unsigned char* halo_ke;    // per node: 0 if another rank counts its kinetic energy
  const unsigned char* xbuf;       // nranks exchange buffers, xbytes each (halo_pack_kernel layout)
  size_t xbytes;
  int nranks, nhalo;
  // rigid links: for a node with code bit 6, link_mean[link_of[n]] replaces its
  // acceleration in the link's directions; null without links
  const int* link_of;
  const LinkMean* link_mean;
  // skewed /BCS: for a node with code bit 7, the fixed directions are those of
  // skew frame skew_of[n] (9 values: x', y', z'); null without skewed BCs
  const int* skew_of;
  const R* skews;
  // rigid bodies: nodes with a nonzero role are updated by rbody_kernel and left
  // out of this pass (their kinetic energy too); null without rigid bodies
  const unsigned char* rb_role;
  // rotational nodes, one bit per node (bit n & 31 of word n >> 5): the nodes of a
  // part with rotations whose inertia or rotational velocity is nonzero.  Only
  // these read their moment slots and write VR; for any other node the rotational
  // update would leave VR as it is (zero moment over zero inertia, zero VR) and add
  // no rotational energy.  Null when no part has rotations.
  const unsigned* rotmask;
  // 1 when fewer than half of the nodes are rotational (a solid mesh with a shell
  // skin): VR is then read only for rotational nodes, after their bit.  0: VR is
  // read for every node ahead of the bit, which keeps the latency chain of a
  // one-wave pass short.
  int rot_sparse;
};

// Whether node n carries rotations in the node pass (NodeArgs::rotmask).
template <class R>
__device__ __forceinline__ bool rot_node(const NodeArgs<R>& a, int n) {
  return a.rotmask && ((__ldg(a.rotmask + (n >> 5)) >> (n & 31)) & 1u);
}

// Exchange buffer of one rank: nhalo force sums (R4), nhalo moment sums (R4),
// then the rank's PartAcc of the cycle.
template <class R>
__host__ __device__ inline size_t halo_buffer_bytes(int nhalo) {
  return 2 * (size_t)nhalo * sizeof(typename Vec4<R>::T) + sizeof(PartAcc);
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
// Programmatic dependent launch.  The cycle's kernels alternate element pass ->
// node pass, each launched with programmatic stream serialization, so a kernel's
// blocks can start while the previous kernel is still running.  Every kernel
//  - issues first the loads that do not depend on the previous kernel (data written
//    two kernels back or earlier, or static),
//  - then pdl_wait(): returns once the previous grid has completed and its writes
//    are visible (immediately when launched without the attribute),
//  - then pdl_trigger(), so the next kernel may start its own prologue.
// Because each kernel triggers only after its wait, the grid two kernels back has
// completed whenever a kernel starts: its prologue may read that grid's output.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// BCS1V (bcs1.F): zero the components of (x, y, z) along the fixed directions of
// code lcod (4 = x, 2 = y, 1 = z) of skew frame sk (rows x', y', z'), projecting
// them out in the reference's order
template <class R>
__device__ inline void bcs1v_skew(int lcod, const R* sk, R& x, R& y, R& z) {
  if (!lcod) return;
  if (lcod == 7) { x = y = z = R(0); return; }
  auto proj = [&](int r) {
    const R s0 = sk[3 * r], s1 = sk[3 * r + 1], s2 = sk[3 * r + 2];
    const R aa = s0 * x + s1 * y + s2 * z;
    x = x - s0 * aa; y = y - s1 * aa; z = z - s2 * aa;
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

// FINTER (tools/curve/finter.F): first segment whose right end is >= xx (the last
// one beyond the end), linear inside and beyond both ends, evaluated from the
// nearer end of the segment; a one-point function is constant
template <class R>
__device__ inline R finter(const double* fx, const double* fy, int n, R xx) {
  if (n == 1) return R(fy[0]);
  R dx2 = R(fx[0]) - xx;
  for (int i = 1; i < n; ++i) {
    const R dx1 = -dx2;
    dx2 = R(fx[i]) - xx;
    if (dx2 >= R(0) || i == n - 1) {
      const R div0 = R(fx[i]) - R(fx[i - 1]);
      R div = fabs(div0) > R(1e-16) ? fabs(div0) : R(1e-16);
      div = div0 >= R(0) ? div : -div;
      const R deri = (R(fy[i]) - R(fy[i - 1])) / div;
      return dx1 <= dx2 ? R(fy[i - 1]) + dx1 * deri : R(fy[i]) - dx2 * deri;
    }
  }
  return R(0);
}

__device__ inline void raise_error(ErrorWord* e, int code, int index) {
  if (atomicCAS(&e->code, 0, code) == 0) e->index = index;
}

__device__ inline unsigned long long dt_key(double dt, int type, int elem) {
  float f = (float)dt;
  unsigned long long hi = (unsigned long long)__float_as_uint(f);
  unsigned lo = (type == 3 ? 0u : 0x80000000u) | (unsigned)elem;
  return (hi << 32) | lo;
}

template <class R> __device__ inline R rsqrt_(R x);
template <class R> __device__ inline R ssqrt(R x) { return sqrt(x); }
__device__ inline float ssqrt(float x) { return sqrtf(x); }

template <class R> __device__ inline R cbrt_(R x) { return cbrt(x); }
__device__ inline float cbrt_(float x) { return cbrtf(x); }
template <class R> __device__ inline R pow_(R x, R y) { return pow(x, y); }
__device__ inline float pow_(float x, float y) { return powf(x, y); }
template <class R> __device__ inline R exp_(R x) { return exp(x); }
__device__ inline float exp_(float x) { return expf(x); }
template <class R> __device__ inline R log_(R x) { return log(x); }
__device__ inline float log_(float x) { return logf(x); }

// block-wide min of a 64-bit key and sums of two doubles (TILE threads)
template <int TILE>
__device__ inline void block_reduce(unsigned long long& key, unsigned long long& bits, double& s0, double& s1,
                                    unsigned long long* skey, unsigned long long* sbits, double* ss0, double* ss1) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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

// ===========================================================================
// register budgets of the patch kernels
// ===========================================================================
// Resident 128-thread CTAs per SM each patch kernel is compiled for (the
// minimum-blocks argument of __launch_bounds__, scaled to the tile).  The
// kernels are issue/latency-bound, so more resident warps pay for a few spilled
// registers (which stay in L1); the defaults are the fastest caps of a sweep on
// B200: hexa FP32 7 CTAs (72 registers; C4 hexa pass 200.6 us against 210.8 at 6
// and 219.5 at 5), shell FP32 3 (168), hexa FP64 4 (128), shell FP64 3 (168).
#ifndef ORB_HEX_CTAS_F32
#define ORB_HEX_CTAS_F32 7
#endif
#ifndef ORB_SHELL_CTAS_F32
#define ORB_SHELL_CTAS_F32 3
#endif
#ifndef ORB_HEX_CTAS_F64
#define ORB_HEX_CTAS_F64 4
#endif
#ifndef ORB_SHELL_CTAS_F64
#define ORB_SHELL_CTAS_F64 3
#endif
// The 5-point shell kernel with its integration-point state staged in shared memory
// holds 30 fewer registers per thread: 5 CTAs (102 registers, 152 B spilled) ran
// C3's shell pass in 221.2 us against 233.5 at 4 CTAs and 256.3 at 3, and 259.3 for
// the register-held form at 3.  It is the form for meshes of more than one wave of
// the register-held kernel; a single wave (the C2 plate at tile 64: 8.0 against
// 8.9 us) keeps the register-held form, whose chain is shorter.
#ifndef ORB_SHELL_STAGED_CTAS_F32
#define ORB_SHELL_STAGED_CTAS_F32 5
#endif
// The 5-point rule of COQINI (coqini.F:45-130) as compile-time constants for the
// NPT = 5 shell kernels (row 0: Z0, 1: WF, 2: WM); the host build checks them
// against the shared table of coqini_table.h.
__host__ __device__ constexpr float coq5(int row, int ip) {
  return row == 0 ? (ip == 0 ? -.5f : ip == 1 ? -.25f : ip == 2 ? 0.f : ip == 3 ? .25f : .5f)
         : row == 1 ? (ip == 0 || ip == 4 ? .125f : .25f)
                    : (ip == 0 ? -.0520833f : ip == 1 ? -.0625f : ip == 2 ? 0.f : ip == 3 ? .0625f : .0520833f);
}

template <class R> struct Occupancy;
template <> struct Occupancy<float> {
  static constexpr int hex = ORB_HEX_CTAS_F32, shell = ORB_SHELL_CTAS_F32, shell_staged = ORB_SHELL_STAGED_CTAS_F32;
};
template <> struct Occupancy<double> {
  static constexpr int hex = ORB_HEX_CTAS_F64, shell = ORB_SHELL_CTAS_F64, shell_staged = ORB_SHELL_CTAS_F64;
};
__host__ __device__ constexpr int min_blocks(int ctas128, int tile) {
  return ctas128 * 128 / tile > 0 ? ctas128 * 128 / tile : 1;
}

// ===========================================================================
// asynchronous copies into shared memory
// ===========================================================================
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// one-arrival mbarrier of a CTA, made visible to the async proxy
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// the arrival, announcing the bytes the bulk copies below will deliver
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// bulk copy (TMA, untiled) of bytes from global to shared memory, completing on bar;
// both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// waits for the phase of bar with the given parity to complete, at most `tries`
// polls; false if it did not
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int tries) {
  unsigned done = 0;
  for (int i = 0; i < tries && !done; ++i)
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
                 : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return done != 0;
}
__device__ __forceinline__ bool mbar_wait0(unsigned long long* bar, int tries) { return mbar_wait(bar, 0u, tries); }
// element-wise asynchronous copies (no register staging), completed by cp_async_wait_all
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// polls of a CTA's staging mbarrier before it reports OR_E_TIMEOUT; its bulk copies
// read this GPU's own memory and complete in microseconds
constexpr int STAGE_WAIT_TRIES = 1 << 22;

// minimum of a 64-bit unsigned value over the warp, from two 32-bit hardware
// reductions (high words, then the low words of the lanes holding the high minimum)
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
  const unsigned hi = __reduce_min_sync(0xffffffffu, (unsigned)(v >> 32));
  const unsigned lo = __reduce_min_sync(0xffffffffu, (unsigned)(v >> 32) == hi ? (unsigned)v : 0xffffffffu);
  return ((unsigned long long)hi << 32) | lo;
}

// ===========================================================================
// hexa patch kernel
// ===========================================================================
// Shared memory of a hexa patch (R = element precision, NLM = nlmax, TILE elements),
// in this order, every block 16-byte aligned:
//   24 corner-force planes of TILE R; planes 0..10 first receive the patch's element
//      state (sig 1..6, eint, rho, qvis, vol0, pla), each thread reading only its own
//      entries before it writes its own corners there
//   conn (uint4) | elem_id (int) | vol0dp (double, split form only)   TILE each
//   node x, y (double2) | node velocity (R4)                           NLM each
//   incidence lists (uint16, inc_stride, a multiple of 8)
//   node z (double)                                                    NLM
template <class R>
__host__ __device__ inline size_t hex_smem_bytes(int nl, int tile, int inc_stride) {
  const bool split = sizeof(R) == 4;
  return 24 * (size_t)tile * sizeof(R) + (size_t)tile * (16 + 4 + (split ? 8 : 0)) +
         (size_t)nl * (16 + 4 * sizeof(R) + 8) + 2 * (size_t)inc_stride;
}

// Per element (thread): SCOOR3, SDERI3, SDLEN3, SDEFO3, SRHO3, SROTA3, MMAIN ->
// M1LAW / M2LAW -> MQVISCB, SHVIS3, SFINT3; corner forces into shared memory.
// CORO = 1: groups may use the convected frame (JCVT /= 0, decided per group at
// run time); CORO = 0 compiles that path out (the register budget of the default)
template <class R, int TILE, int CORO>
__global__ void __launch_bounds__(TILE, min_blocks(Occupancy<R>::hex, TILE))
hex_patch_kernel(HexArgs<R> a, int parity) {
  typedef typename Vec4<R>::T R4;
  constexpr bool split = sizeof(R) == 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned long long s_key[TILE / 32], s_bits[TILE / 32];
  __shared__ double s_s0[TILE / 32], s_s1[TILE / 32];
  __shared__ __align__(8) unsigned long long s_bar;
  __shared__ __align__(16) HexGroupDesc s_gd;
  const int p = blockIdx.x;
  const int tid = threadIdx.x;
  // Patches are padded to TILE elements (element p*TILE + t is thread t's) and their
  // node lists to nlmax entries, so every address below follows from (p, tid) alone.
  const int NLM = a.nlmax;
  const int nelpad = a.nelpad;
  const size_t e0 = (size_t)p * TILE;
  const int e = p * TILE + tid;
  R* sc = reinterpret_cast<R*>(smem_raw);
  uint4* sconn = reinterpret_cast<uint4*>(sc + 24 * TILE);
  int* seid = reinterpret_cast<int*>(sconn + TILE);
  double* svol0dp = reinterpret_cast<double*>(seid + TILE);
  double2* sxy = reinterpret_cast<double2*>(svol0dp + (split ? TILE : 0));
  R4* sv = reinterpret_cast<R4*>(sxy + NLM);
  unsigned short* sinc = reinterpret_cast<unsigned short*>(sv + NLM);
  double* sz = reinterpret_cast<double*>(sinc + a.inc_stride);
  // One thread stages the patch's element state, connectivity and incidence lists by
  // bulk copies.  They were written two launches back or are static, so they are
  // issued before the wait on the previous kernel (the node pass).
  if (tid == 0) {
    mbar_init(&s_bar);
    const unsigned pl = TILE * sizeof(R);
    mbar_expect_tx(&s_bar, 11 * pl + TILE * (16 + 4 + (split ? 8 : 0)) + 2 * a.inc_stride +
                               (unsigned)sizeof(HexGroupDesc));
#pragma unroll
    for (int c = 0; c < 6; ++c) bulk_g2s(sc + c * TILE, a.sig + (size_t)c * nelpad + e0, pl, &s_bar);
    bulk_g2s(sc + 6 * TILE, a.eint + e0, pl, &s_bar);
    bulk_g2s(sc + 7 * TILE, a.rho + e0, pl, &s_bar);
    bulk_g2s(sc + 8 * TILE, a.qvis + e0, pl, &s_bar);
    bulk_g2s(sc + 9 * TILE, a.vol0 + e0, pl, &s_bar);
    bulk_g2s(sc + 10 * TILE, a.pla + e0, pl, &s_bar);
    bulk_g2s(sconn, a.conn + e0, TILE * 16, &s_bar);
    bulk_g2s(seid, a.elem_id + e0, TILE * 4, &s_bar);
    if (split) bulk_g2s(svol0dp, a.vol0dp + e0, TILE * 8, &s_bar);
    bulk_g2s(sinc, a.inc + (size_t)p * a.inc_stride, 2 * a.inc_stride, &s_bar);
  }
  const PatchInfo pi = a.patch[p];
  // the patch's group constants, staged too (the byte count above includes them)
  if (tid == 0) bulk_g2s(&s_gd, a.groups + pi.group, sizeof(HexGroupDesc), &s_bar);
  // issued now, used at the end: the patch's slot numbers (up to two per thread)
  // and its cumulative energy partials
  const int slot0 = tid < NLM ? a.patch_slots[p * NLM + tid] : -1;
  const int slot1 = tid + TILE < NLM ? a.patch_slots[p * NLM + tid + TILE] : -1;
  double pre_ehour = 0.0, pre_wpla = 0.0;
  if (tid == 0) { pre_ehour = a.blk_ehour[p]; pre_wpla = a.blk_wpla[p]; }
  // X, V and the cycle's time come from the previous node pass: gathered after the
  // wait, straight into shared memory
  pdl_wait();
  pdl_trigger();
  for (int j = tid; j < NLM; j += TILE) {
    const int g = a.patch_nodes[p * NLM + j];
    const double* xg = reinterpret_cast<const double*>(a.X + g);
    cp_async16(sxy + j, xg);
    cp_async8(sz + j, xg + 2);
    if (split) {
      cp_async16(sv + j, a.V + g);
    } else {
      cp_async16(sv + j, a.V + g);
      cp_async16(reinterpret_cast<unsigned char*>(sv + j) + 16, reinterpret_cast<const unsigned char*>(a.V + g) + 16);
    }
  }
  const bool active = tid < pi.nel;
  const int nl = pi.nloc;
  const PartTime& tm = a.time[parity * a.nparts + pi.part];
  const R DT1 = R(tm.dt2);
  cp_async_wait_all();
  __syncthreads();   // node gathers of every thread landed; the mbarrier is initialised
  if (!mbar_wait0(&s_bar, STAGE_WAIT_TRIES)) raise_error(a.err, 7, p);

  unsigned long long mykey = ~0ull, mybits = ~0ull;
  double my_ehou = 0.0, my_wpla = 0.0;
  if (active) {
    const uint4 cw = sconn[tid];
    // local node of corner k (the colour bits of corner 0 masked off)
    auto corner = [&](int k) -> int {
      const unsigned w = k < 2 ? cw.x : k < 4 ? cw.y : k < 6 ? cw.z : cw.w;
      const int l = (k & 1) ? (int)(w >> 16) : (int)(w & 0xffffu);
      return k == 0 ? (l & (int)LOCAL_MASK) : l;
    };
    const int st_eid = seid[tid];
    // ---- SDERI3 in FP64 (sderi3.F:103-149, 264-298): the corner differences of the
    // pairs 1-7, 2-8, 3-5, 4-6, and the coordinates relative to corner 1 (differences
    // taken in FP64, then rounded to R: beyond the determinant nothing needs FP64, as in
    // the reference's -prec=sp build, which forms the inverse Jacobian, the hourglass
    // vectors and SDLEN3 in my_real) ----
    double X17, X28, X35, X46, Y17, Y28, Y35, Y46, Z17, Z28, Z35, Z46;
    R xr[8], yr[8], zr[8];
    R R11 = R(1), R12 = R(0), R13 = R(0), R21 = R(0), R22 = R(1), R23 = R(0), R31 = R(0), R32 = R(0), R33 = R(1);
    const bool corot = CORO && s_gd.jcvt;
    if (corot) {
      double XD[8], YD[8], ZD[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int l = corner(k);
        const double2 xy = sxy[l];
        XD[k] = xy.x; YD[k] = xy.y; ZD[k] = sz[l];
      }
      // SRCOOR3 (srcoor3.F, JCVT /= 0, ISORTH = 0): convected frame R = [e1 e2 e3] of
      // SREPISO3 (FP64 differences, r, s, t in R) and SORTHO3 (three symmetric
      // corrections, then Gram-Schmidt); coordinates (FP64) and velocities in it
      const R x17 = R(XD[6] - XD[0]), x28 = R(XD[7] - XD[1]), x35 = R(XD[4] - XD[2]), x46 = R(XD[5] - XD[3]);
      const R y17 = R(YD[6] - YD[0]), y28 = R(YD[7] - YD[1]), y35 = R(YD[4] - YD[2]), y46 = R(YD[5] - YD[3]);
      const R z17 = R(ZD[6] - ZD[0]), z28 = R(ZD[7] - ZD[1]), z35 = R(ZD[4] - ZD[2]), z46 = R(ZD[5] - ZD[3]);
      const R a17 = x17 + x46, a28 = x28 + x35, b17 = y17 + y46, b28 = y28 + y35, c17 = z17 + z46, c28 = z28 + z35;
      R Ux = x17 + x28 - x35 - x46, Uy = y17 + y28 - y35 - y46, Uz = z17 + z28 - z35 - z46;
      R Vx = a17 + a28, Vy = b17 + b28, Vz = c17 + c28;
      R Wx = a17 - a28, Wy = b17 - b28, Wz = c17 - c28;
      auto unit = [](R& x, R& y, R& z) {
        R aa = ssqrt(x * x + y * y + z * z);
        if (aa != R(0)) aa = R(1) / aa;
        x *= aa; y *= aa; z *= aa;
      };
      unit(Ux, Uy, Uz); unit(Vx, Vy, Vz); unit(Wx, Wy, Wz);
#pragma unroll
      for (int it = 0; it < 3; ++it) {
        R e1x = Vy * Wz - Vz * Wy + Ux, e1y = Vz * Wx - Vx * Wz + Uy, e1z = Vx * Wy - Vy * Wx + Uz;
        R e2x = Wy * Uz - Wz * Uy + Vx, e2y = Wz * Ux - Wx * Uz + Vy, e2z = Wx * Uy - Wy * Ux + Vz;
        R e3x = Uy * Vz - Uz * Vy + Wx, e3y = Uz * Vx - Ux * Vz + Wy, e3z = Ux * Vy - Uy * Vx + Wz;
        unit(e1x, e1y, e1z); unit(e2x, e2y, e2z); unit(e3x, e3y, e3z);
        Ux = e1x; Uy = e1y; Uz = e1z; Vx = e2x; Vy = e2y; Vz = e2z; Wx = e3x; Wy = e3y; Wz = e3z;
      }
      R e3x = Uy * Vz - Uz * Vy, e3y = Uz * Vx - Ux * Vz, e3z = Ux * Vy - Uy * Vx;
      unit(e3x, e3y, e3z);
      R11 = Ux; R21 = Uy; R31 = Uz;
      R12 = e3y * Uz - e3z * Uy; R22 = e3z * Ux - e3x * Uz; R32 = e3x * Uy - e3y * Ux;
      R13 = e3x; R23 = e3y; R33 = e3z;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const double xl = (double)R11 * XD[k] + (double)R21 * YD[k] + (double)R31 * ZD[k];
        const double yl = (double)R12 * XD[k] + (double)R22 * YD[k] + (double)R32 * ZD[k];
        const double zl = (double)R13 * XD[k] + (double)R23 * YD[k] + (double)R33 * ZD[k];
        XD[k] = xl; YD[k] = yl; ZD[k] = zl;
      }
      X17 = XD[6] - XD[0]; X28 = XD[7] - XD[1]; X35 = XD[4] - XD[2]; X46 = XD[5] - XD[3];
      Y17 = YD[6] - YD[0]; Y28 = YD[7] - YD[1]; Y35 = YD[4] - YD[2]; Y46 = YD[5] - YD[3];
      Z17 = ZD[6] - ZD[0]; Z28 = ZD[7] - ZD[1]; Z35 = ZD[4] - ZD[2]; Z46 = ZD[5] - ZD[3];
#pragma unroll
      for (int k = 0; k < 8; ++k) { xr[k] = R(XD[k] - XD[0]); yr[k] = R(YD[k] - YD[0]); zr[k] = R(ZD[k] - ZD[0]); }
    } else {
      // corner 1 first, then the pairs, so that at most two corners are held in FP64
      const int l0 = corner(0);
      const double2 q0 = sxy[l0];
      const double x0 = q0.x, y0 = q0.y, z0 = sz[l0];
      xr[0] = R(0); yr[0] = R(0); zr[0] = R(0);
      auto ld = [&](int k, double& x, double& y, double& z) {
        const int l = corner(k);
        const double2 q = sxy[l];
        x = q.x; y = q.y; z = sz[l];
        xr[k] = R(x - x0); yr[k] = R(y - y0); zr[k] = R(z - z0);
      };
      double xk, yk, zk, xm, ym, zm;
      ld(6, xk, yk, zk);
      X17 = xk - x0; Y17 = yk - y0; Z17 = zk - z0;
      ld(1, xm, ym, zm); ld(7, xk, yk, zk);
      X28 = xk - xm; Y28 = yk - ym; Z28 = zk - zm;
      ld(2, xm, ym, zm); ld(4, xk, yk, zk);
      X35 = xk - xm; Y35 = yk - ym; Z35 = zk - zm;
      ld(3, xm, ym, zm); ld(5, xk, yk, zk);
      X46 = xk - xm; Y46 = yk - ym; Z46 = zk - zm;
    }
    const double J1 = X17 + X28 - X35 - X46, J2 = Y17 + Y28 - Y35 - Y46, J3 = Z17 + Z28 - Z35 - Z46;
    const double xa = X17 + X46, xb = X28 + X35, ya = Y17 + Y46, yb = Y28 + Y35, za = Z17 + Z46, zb = Z28 + Z35;
    const double J4 = xa + xb, J5 = ya + yb, J6 = za + zb, J7 = xa - xb, J8 = ya - yb, J9 = za - zb;
    const double C1 = J5 * J9 - J6 * J8, C4 = J6 * J7 - J4 * J9, C7 = J4 * J8 - J5 * J7;
    double det = (1.0 / 64.0) * (J1 * C1 + J2 * C4 + J3 * C7);
    if (!(det > 0.0)) {   // SCHKJABT3: zero or negative volume stops the run
      raise_error(a.err, 4, st_eid);
      det = 1.0;
    }
    const R j1 = R(J1), j2 = R(J2), j3 = R(J3), j4 = R(J4), j5 = R(J5), j6 = R(J6), j7 = R(J7), j8 = R(J8), j9 = R(J9);
    const R dett = R(1.0 / 64.0) / R(det);
    const R I1 = dett * R(C1), I4 = dett * R(C4), I7 = dett * R(C7);
    const R I2 = dett * (j3 * j8 - j2 * j9), I5 = dett * (j1 * j9 - j3 * j7), I8 = dett * (j2 * j7 - j1 * j8);
    const R I3 = dett * (j2 * j6 - j3 * j5), I6 = dett * (j3 * j4 - j1 * j6), I9 = dett * (j1 * j5 - j2 * j4);
    R PX[4], PY[4], PZ[4];
    {
      const R a12 = I1 + I2, a45 = I4 + I5, a78 = I7 + I8;
      const R b12 = I1 - I2, b45 = I4 - I5, b78 = I7 - I8;
      PX[0] = -a12 - I3; PY[0] = -a45 - I6; PZ[0] = -a78 - I9;
      PX[1] = -a12 + I3; PY[1] = -a45 + I6; PZ[1] = -a78 + I9;
      PX[2] = b12 + I3;  PY[2] = b45 + I6;  PZ[2] = b78 + I9;
      PX[3] = b12 - I3;  PY[3] = b45 - I6;  PZ[3] = b78 - I9;
    }
    // hourglass projections PXiHj (sderi3.F:302-333): modes (+-+-+-+-), (++----++), (+--+-++-);
    // the mode vectors sum to zero, so relative coordinates give the same products
    R PXH[4][3];
    {
      const R hx1 = xr[0] - xr[1] + xr[2] - xr[3] + xr[4] - xr[5] + xr[6] - xr[7];
      const R hy1 = yr[0] - yr[1] + yr[2] - yr[3] + yr[4] - yr[5] + yr[6] - yr[7];
      const R hz1 = zr[0] - zr[1] + zr[2] - zr[3] + zr[4] - zr[5] + zr[6] - zr[7];
      const R hx2 = xr[0] + xr[1] - xr[2] - xr[3] - xr[4] - xr[5] + xr[6] + xr[7];
      const R hy2 = yr[0] + yr[1] - yr[2] - yr[3] - yr[4] - yr[5] + yr[6] + yr[7];
      const R hz2 = zr[0] + zr[1] - zr[2] - zr[3] - zr[4] - zr[5] + zr[6] + zr[7];
      const R hx3 = xr[0] - xr[1] - xr[2] + xr[3] - xr[4] + xr[5] + xr[6] - xr[7];
      const R hy3 = yr[0] - yr[1] - yr[2] + yr[3] - yr[4] + yr[5] + yr[6] - yr[7];
      const R hz3 = zr[0] - zr[1] - zr[2] + zr[3] - zr[4] + zr[5] + zr[6] - zr[7];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        PXH[q][0] = PX[q] * hx1 + PY[q] * hy1 + PZ[q] * hz1;
        PXH[q][1] = PX[q] * hx2 + PY[q] * hy2 + PZ[q] * hz2;
        PXH[q][2] = PX[q] * hx3 + PY[q] * hy3 + PZ[q] * hz3;
      }
    }
    const double VOLN_D = det;
    const R VOLN = R(det);
    // ---- SDLEN3 / SLEN (sdlen3.F:110-166): 4 V / sqrt(max face (E G - F^2)) ----
    R AREAM = R(EM20);
    {
      const int FC[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const R x13 = xr[FC[f][2]] - xr[FC[f][0]], x24 = xr[FC[f][3]] - xr[FC[f][1]];
        const R y13 = yr[FC[f][2]] - yr[FC[f][0]], y24 = yr[FC[f][3]] - yr[FC[f][1]];
        const R z13 = zr[FC[f][2]] - zr[FC[f][0]], z24 = zr[FC[f][3]] - zr[FC[f][1]];
        const R s1 = x13 - x24, t1 = x13 + x24, s2 = y13 - y24, t2 = y13 + y24, s3 = z13 - z24, t3 = z13 + z24;
        const R E = s1 * s1 + s2 * s2 + s3 * s3, Fm = s1 * t1 + s2 * t2 + s3 * t3, G = t1 * t1 + t2 * t2 + t3 * t3;
        const R ar = E * G - Fm * Fm;
        AREAM = ar > AREAM ? ar : AREAM;
      }
    }
    const R DELTAX = R(4) * VOLN / ssqrt(AREAM);
    // ---- SDEFO3 (sdefo3.F:114-170, JHBE=1) and the hourglass velocity modes of
    // SHVIS3, from the velocities taken in the corner pairs (1,7) (2,8) (3,5) (4,6)
    // that share a row of PX: the mode-j sum  sum_k g_jk v_k  with g_jk = s_jk -+ PXH
    // splits into the sign sum  sum_k s_jk v_k  and  -sum_q PXH[q][j] (v_k1 - v_k2) ----
    constexpr int sgn[3][8] = {{1, -1, 1, -1, 1, -1, 1, -1}, {1, 1, -1, -1, -1, -1, 1, 1}, {1, -1, -1, 1, -1, 1, 1, -1}};
    constexpr int h4[8] = {1, -1, 1, -1, -1, 1, -1, 1};
    constexpr int pk1[4] = {0, 1, 2, 3}, pk2[4] = {6, 7, 4, 5};
    R DXX = R(0), DYY = R(0), DZZ = R(0), DXY = R(0), DXZ = R(0), DYX = R(0), DYZ = R(0), DZX = R(0), DZY = R(0);
    R HGX[4] = {R(0), R(0), R(0), R(0)}, HGY[4] = {R(0), R(0), R(0), R(0)}, HGZ[4] = {R(0), R(0), R(0), R(0)};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k1 = pk1[q], k2 = pk2[q];
      const R4 v1 = sv[corner(k1)], v2 = sv[corner(k2)];
      R u1 = v1.x, w1 = v1.y, t1 = v1.z, u2 = v2.x, w2 = v2.y, t2 = v2.z;
      if (corot) {
        const R a1 = R11 * u1 + R21 * w1 + R31 * t1, b1 = R12 * u1 + R22 * w1 + R32 * t1, c1 = R13 * u1 + R23 * w1 + R33 * t1;
        const R a2 = R11 * u2 + R21 * w2 + R31 * t2, b2 = R12 * u2 + R22 * w2 + R32 * t2, c2 = R13 * u2 + R23 * w2 + R33 * t2;
        u1 = a1; w1 = b1; t1 = c1; u2 = a2; w2 = b2; t2 = c2;
      }
      const R dvx = u1 - u2, dvy = w1 - w2, dvz = t1 - t2;
      DXX += PX[q] * dvx; DYY += PY[q] * dvy; DZZ += PZ[q] * dvz;
      DXY += PY[q] * dvx; DXZ += PZ[q] * dvx; DYX += PX[q] * dvy;
      DYZ += PZ[q] * dvy; DZX += PX[q] * dvz; DZY += PY[q] * dvz;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const R s1 = R(sgn[j][k1]), s2 = R(sgn[j][k2]);
        HGX[j] += s1 * u1 + s2 * u2 - PXH[q][j] * dvx;
        HGY[j] += s1 * w1 + s2 * w2 - PXH[q][j] * dvy;
        HGZ[j] += s1 * t1 + s2 * t2 - PXH[q][j] * dvz;
      }
      // the 4th mode (+-+--+-+) (shvis3.F:230-232)
      HGX[3] += R(h4[k1]) * u1 + R(h4[k2]) * u2;
      HGY[3] += R(h4[k1]) * w1 + R(h4[k2]) * w2;
      HGZ[3] += R(h4[k1]) * t1 + R(h4[k2]) * t2;
    }
    // PXH is needed again only by SFINT3: parked in this thread's own entries of the
    // corner planes 11..22 (free until its corners are written; volatile, so that the
    // compiler reloads them instead of holding 12 registers across the material law)
    volatile R* park = sc + 11 * TILE + tid;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int j = 0; j < 3; ++j) park[(3 * q + j) * TILE] = PXH[q][j];
    const R DT1D2 = R(0.5) * DT1;
    const R D4 = DXY + DYX, D5 = DYZ + DZY, D6 = DXZ + DZX;
    const R WZZ = DT1D2 * (DYX - DXY), WYY = DT1D2 * (DXZ - DZX), WXX = DT1D2 * (DZY - DYZ);
    // ---- SRHO3 (srho3.F:122-156; FP64 volume ratios in the split form, srho3.F:230-245) ----
    const R RHO0 = R(s_gd.rho0);
    const R rho_old = sc[7 * TILE + tid];
    const R VOLO = sc[9 * TILE + tid];
    R DVOL, RHON, AMU;
    if (split) {
      const double v0 = svol0dp[tid];
      DVOL = R(VOLN_D - ((double)RHO0 / (double)rho_old) * v0);
      RHON = R((double)RHO0 * (v0 / VOLN_D));
      AMU = R(v0 / VOLN_D - 1.0);
    } else {
      DVOL = VOLN - (RHO0 / rho_old) * VOLO;
      RHON = RHO0 * (VOLO / VOLN);
      AMU = RHON / RHO0 - R(1);
    }
    R EINT = sc[6 * TILE + tid] * VOLO;
    // ---- SROTA3 Jaumann rotation (srota3.F:81-91) ----
    const R S1 = sc[0 * TILE + tid], S2 = sc[1 * TILE + tid], S3 = sc[2 * TILE + tid];
    const R S4 = sc[3 * TILE + tid], S5 = sc[4 * TILE + tid], S6 = sc[5 * TILE + tid];
    R SG[6];
    if (corot) {          // SRMALLA3 (srmall3.F): convected-frame stress, not rotated
      SG[0] = S1; SG[1] = S2; SG[2] = S3; SG[3] = S4; SG[4] = S5; SG[5] = S6;
    } else {
      const R q1 = R(2) * S4 * WZZ, q2 = R(2) * S6 * WYY, q3 = R(2) * S5 * WXX;
      SG[0] = S1 - q1 + q2;
      SG[1] = S2 + q1 - q3;
      SG[2] = S3 - q2 + q3;
      SG[3] = S4 + WZZ * (S1 - S2) + WYY * S5 - WXX * S6;
      SG[4] = S5 + WXX * (S2 - S3) + WZZ * S6 - WYY * S4;
      SG[5] = S6 + WYY * (S3 - S1) + WXX * S4 - WZZ * S5;
    }
    const R VOL_AVG = VOLN - R(0.5) * DVOL;
    const R QOLD = sc[8 * TILE + tid];
    const R EPXE = sc[10 * TILE + tid];
    // the state planes 0..10 are read: PX, PY, PZ (needed again only by SFINT3) are
    // parked in this thread's entries of planes 0..10 and 23 likewise
    volatile R* park2 = sc + tid;
    constexpr int pplane[12] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 23};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      park2[pplane[q] * TILE] = PX[q];
      park2[pplane[4 + q] * TILE] = PY[q];
      park2[pplane[8 + q] * TILE] = PZ[q];
    }
    // ---- elastic predictor (m1law.F:124-140 / m2law.F:187-200) ----
    const R OFF = R(1);
    const R Gs = R(s_gd.shear) * OFF;
    const R G1 = DT1 * Gs, G2 = R(2) * G1;
    const R SSP = ssqrt((R(1.333) * Gs + R(s_gd.bulk)) / RHO0);
    {
      const R P = -R(1.0 / 3.0) * (SG[0] + SG[1] + SG[2]);
      const R DAV = -R(1.0 / 3.0) * (DXX + DYY + DZZ);
      SG[0] = SG[0] + P + G2 * (DXX + DAV);
      SG[1] = SG[1] + P + G2 * (DYY + DAV);
      SG[2] = SG[2] + P + G2 * (DZZ + DAV);
      SG[3] = SG[3] + G1 * D4;
      SG[4] = SG[4] + G1 * D5;
      SG[5] = SG[5] + G1 * D6;
    }
    R DPLA = R(0), SIGY = R(0);
    if (s_gd.law == 2) {
      // ---- M2LAW radial return (m2law.F:197-352), CC=0, FISOKIN=0 ----
      R AJ2 = R(0.5) * (SG[0] * SG[0] + SG[1] * SG[1] + SG[2] * SG[2]) + SG[3] * SG[3] + SG[4] * SG[4] + SG[5] * SG[5];
      AJ2 = ssqrt(R(3) * AJ2);
      {   // MSTRAIN_RATE, ISRATE = 0, total strain rate
        const R e4 = R(0.5) * D4, e5 = R(0.5) * D5, e6 = R(0.5) * D6;
        a.epsd[e] = ssqrt(DXX * DXX + DYY * DYY + DZZ * DZZ + R(2) * (e4 * e4 + e5 * e5 + e6 * e6));
      }
      const R CA = R(s_gd.jc_a), CB = R(s_gd.jc_b), CN = R(s_gd.jc_n);
      R AK, QH;
      if (CN == R(1)) { AK = CA + CB * EPXE; QH = CB; }
      else if (EPXE > R(0)) {
        AK = CA + CB * pow_(EPXE, CN);
        QH = (CN > R(1)) ? CB * CN * pow_(EPXE, CN - R(1)) : CB * CN / pow_(EPXE, R(1) - CN);
      } else { AK = CA; QH = R(0); }
      if (R(s_gd.sigmax) < AK) { AK = R(s_gd.sigmax); QH = R(0); }
      SIGY = AK;
      if (EPXE > R(s_gd.epsmax)) { AK = R(0); QH = R(0); }
      R SCALE = AK / (AJ2 > R(EM15) ? AJ2 : R(EM15));
      SCALE = SCALE < R(1) ? SCALE : R(1);
      const R den = R(3) * Gs + QH;
      DPLA = (R(1) - SCALE) * AJ2 / (den > R(EM15) ? den : R(EM15));
      AK = AK + DPLA * QH;
      SCALE = AK / (AJ2 > R(EM15) ? AJ2 : R(EM15));
      SCALE = SCALE < R(1) ? SCALE : R(1);
#pragma unroll
      for (int c = 0; c < 6; ++c) SG[c] = SCALE * SG[c];
      a.pla[e] = EPXE + DPLA;
      SIGY = SIGY > AK ? SIGY : AK;
    }
    // ---- MQVISCB (mqviscb.F:139-354) ----
    R QNEW;
    const R AL = VOLN > R(0) ? cbrt_(VOLN) : R(0);
    {
      const R DD = -DXX - DYY - DZZ;
      const R AD = DD > R(0) ? DD : R(0);
      const R QA = R(s_gd.qa), QB = R(s_gd.qb);
      const R QAA = QA * QA * AD;
      const R QX = QB * SSP + AL * QAA;
      QNEW = RHON * AD * AL * (QAA * AL + QB * SSP);
      R SSP_EQ = QX + ssqrt(QX * QX + SSP * SSP);
      SSP_EQ = SSP_EQ > R(EM20) ? SSP_EQ : R(EM20);
      const R DTX = R(s_gd.dtfac) * (DELTAX / SSP_EQ);
      if ((double)DTX <= s_gd.dtmin) raise_error(a.err, 5, st_eid);
      const double dtd = (double)DTX;
      mykey = dt_key(dtd, 1, st_eid);
      mybits = (unsigned long long)__double_as_longlong(dtd);
    }
    // ---- pressure and internal energy (m1law.F:172-190 / m2law.F:434-461) ----
    const R PNEW = R(s_gd.bulk) * AMU;
    SG[0] = (SG[0] - PNEW) * OFF; SG[1] = (SG[1] - PNEW) * OFF; SG[2] = (SG[2] - PNEW) * OFF;
    SG[3] = SG[3] * OFF; SG[4] = SG[4] * OFF; SG[5] = SG[5] * OFF;
    const R DTA = R(0.5) * DT1;
    R EINC;
    if (s_gd.law == 1) {
      const R P2 = -(S1 + SG[0] + S2 + SG[1] + S3 + SG[2]) * R(1.0 / 3.0);
      EINC = VOL_AVG * (DXX * (S1 + SG[0] + P2) + DYY * (S2 + SG[1] + P2) + DZZ * (S3 + SG[2] + P2) +
                        D4 * (S4 + SG[3]) + D5 * (S5 + SG[4]) + D6 * (S6 + SG[5])) * DTA -
             R(0.5) * DVOL * (QOLD + QNEW + P2);
    } else {
      EINC = VOL_AVG * (DXX * (S1 + SG[0]) + DYY * (S2 + SG[1]) + DZZ * (S3 + SG[2]) +
                        D4 * (S4 + SG[3]) + D5 * (S5 + SG[4]) + D6 * (S6 + SG[5])) * DTA -
             R(0.5) * DVOL * (QOLD + QNEW);
      my_wpla = (double)SIGY * (double)DPLA * (double)VOLN;
    }
    const R vdiv = VOLO > R(EM15) ? VOLO : R(EM15);
    EINT = (EINT + EINC * OFF) / vdiv;
#pragma unroll
    for (int c = 0; c < 6; ++c) a.sig[c * nelpad + e] = SG[c];
    a.eint[e] = EINT;
    a.rho[e] = RHON;
    a.qvis[e] = QNEW;
    // ---- SHVIS3 Flanagan-Belytschko viscous hourglass (shvis3.F:156-424, JHBE>=1) ----
    const R CAQ = R(0.25) * OFF * R(s_gd.qh);
    R FCL = CAQ * RHON * (AL * AL);   // VOL**TWO_THIRD
    const R FCQ = FCL * CAQ * R(100);
    FCL = FCL * SSP;
    R HX[4], HY[4], HZ[4];
    {
      R ehou = R(0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        HX[j] = HGX[j] * (FCL + fabs(HGX[j]) * FCQ);
        HY[j] = HGY[j] * (FCL + fabs(HGY[j]) * FCQ);
        HZ[j] = HGZ[j] * (FCL + fabs(HGZ[j]) * FCQ);
        ehou += HX[j] * HGX[j] + HY[j] * HGY[j] + HZ[j] * HGZ[j];
      }
      my_ehou = (double)(DT1 * ehou);
    }
    // ---- SFINT3 (sfint3.F:256-321), antisymmetric pairs 1-7, 2-8, 3-5, 4-6: corner
    // k1 gets -f_q, corner k2 gets +f_q, added to the hourglass force; the hourglass
    // force  -sum_j g_jk H_j - h4_k H_4  splits like the mode sums above ----
    const R s1 = (SG[0] - QNEW) * VOLN, s2 = (SG[1] - QNEW) * VOLN, s3 = (SG[2] - QNEW) * VOLN;
    const R s4 = SG[3] * VOLN, s5 = SG[4] * VOLN, s6 = SG[5] * VOLN;
    // PXH, PX, PY, PZ back from their parking planes, before any corner is written
    R PH[4][3], QX[4], QY[4], QZ[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
      for (int j = 0; j < 3; ++j) PH[q][j] = park[(3 * q + j) * TILE];
      QX[q] = park2[pplane[q] * TILE];
      QY[q] = park2[pplane[4 + q] * TILE];
      QZ[q] = park2[pplane[8 + q] * TILE];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k1 = pk1[q], k2 = pk2[q];
      // common part of the pair: sum_j PXH[q][j] H_j minus the stress term
      const R ux = PH[q][0] * HX[0] + PH[q][1] * HX[1] + PH[q][2] * HX[2] - (s1 * QX[q] + s4 * QY[q] + s6 * QZ[q]);
      const R uy = PH[q][0] * HY[0] + PH[q][1] * HY[1] + PH[q][2] * HY[2] - (s2 * QY[q] + s4 * QX[q] + s5 * QZ[q]);
      const R uz = PH[q][0] * HZ[0] + PH[q][1] * HZ[1] + PH[q][2] * HZ[2] - (s3 * QZ[q] + s6 * QX[q] + s5 * QY[q]);
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const int k = side ? k2 : k1;
        const R sg = side ? R(-1) : R(1);
        R fx = -R(sgn[0][k]) * HX[0] - R(sgn[1][k]) * HX[1] - R(sgn[2][k]) * HX[2] - R(h4[k]) * HX[3] + sg * ux;
        R fy = -R(sgn[0][k]) * HY[0] - R(sgn[1][k]) * HY[1] - R(sgn[2][k]) * HY[2] - R(h4[k]) * HY[3] + sg * uy;
        R fz = -R(sgn[0][k]) * HZ[0] - R(sgn[1][k]) * HZ[1] - R(sgn[2][k]) * HZ[2] - R(h4[k]) * HZ[3] + sg * uz;
        if (corot) {        // SRROTA3 with R transposed (sforc3.F:1603-1614): back to global axes
          const R gx = R11 * fx + R12 * fy + R13 * fz;
          const R gy = R21 * fx + R22 * fy + R23 * fz;
          const R gz = R31 * fx + R32 * fy + R33 * fz;
          fx = gx; fy = gy; fz = gz;
        }
        // planes 0..10 held this thread's own state, read above
        sc[(0 * 8 + k) * TILE + tid] = fx;
        sc[(1 * 8 + k) * TILE + tid] = fy;
        sc[(2 * 8 + k) * TILE + tid] = fz;
      }
    }
  }
  // ---- patch assembly: each patch node sums its incident corners in ascending
  // (element, corner) order ----
  __syncthreads();
  for (int j = tid; j < nl; j += TILE) {
    R fx = R(0), fy = R(0), fz = R(0);
    const int i1 = sinc[j + 1];
#pragma unroll 4
    for (int i = sinc[j]; i < i1; ++i) {
      const int o = sinc[NLM + 1 + i];     // corner k of element t: k * TILE + t
      fx += sc[o]; fy += sc[8 * TILE + o]; fz += sc[16 * TILE + o];
    }
    const int s = j == tid ? slot0 : j == tid + TILE ? slot1 : a.patch_slots[p * NLM + j];
    a.fslot[s] = mk4(fx, fy, fz, R(0));
  }
  // ---- dt min-reduction and energy partials (fixed tree order for the sums) ----
  {
    const int lane = tid & 31, warp = tid >> 5;
    mykey = warp_min_u64(mykey);
    mybits = warp_min_u64(mybits);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      my_ehou += __shfl_xor_sync(0xffffffffu, my_ehou, o);
      my_wpla += __shfl_xor_sync(0xffffffffu, my_wpla, o);
    }
    if (lane == 0) { s_key[warp] = mykey; s_bits[warp] = mybits; s_s0[warp] = my_ehou; s_s1[warp] = my_wpla; }
    __syncthreads();
    if (tid == 0) {
      unsigned long long k = s_key[0], b = s_bits[0];
      double h = s_s0[0], w = s_s1[0];
#pragma unroll
      for (int i = 1; i < TILE / 32; ++i) {
        k = s_key[i] < k ? s_key[i] : k;
        b = s_bits[i] < b ? s_bits[i] : b;
        h += s_s0[i];
        w += s_s1[i];
      }
      PartAcc* acc = &a.acc[parity * a.nparts + pi.part];
      atomicMin(&acc->dtkey, k);
      atomicMin(&acc->dtbits, b);
      a.blk_ehour[p] = pre_ehour + h;
      a.blk_wpla[p] = pre_wpla + w;
    }
  }
}


// ===========================================================================
// one BT shell element (CFORC3 chain), shared by the patch kernel and the
// persistent kernel
// ===========================================================================
// M2CPLR's iterative returns for a plane-stress point already outside the yield
// surface test (FISOKIN = 0, no rate or thermal term): IPLA = 1, three Newton
// iterations on DPLA with the plane-stress correction factors P, Q
// (m2cplr.F:231-378); IPLA = 2, an approximate normal projection then a radial
// return to the hardened yield stress (m2cplr.F:379-445).  SN: sigma xx, yy, xy
// (updated); PLA, YLD (IPLA 2 hardens it), DPLA, EZZ (the plastic thickness
// strain term, before SIGEPS02C's elastic part) out.  Returns whether the point
// flowed.
template <class R>
__device__ __forceinline__ bool m2cplr_iterative(const int ipla, R (&SN)[5], R& PLA, R& YLD, R& DPLA, R& EZZ,
                                                 const R CA, const R CB, const R CN, const R YMAX, const R YOUNG,
                                                 const R NU, const R G, const R OFF) {
  const R SMALL = R(1e-7);
  if (ipla == 1) {
    const R S1 = SN[0] + SN[1], S2 = SN[0] - SN[1], S3 = SN[2];
    const R A = R(0.25) * S1 * S1;
    const R B = R(0.75) * S2 * S2 + R(3) * S3 * S3;
    const R SVM = ssqrt(A + B);
    if (!(SVM > YLD && OFF == R(1))) return false;
    const R NU1 = R(1) / (R(1) - NU), NU2 = R(1) / (R(1) + NU);
    const R H = YLD >= YMAX ? R(0) : CN * CB * exp_((CN - R(1)) * log_(PLA + SMALL));
    R DPLA_J = (SVM - YLD) / (R(3) * G + H);
    const R ANU1 = A * NU1, BNU2 = R(3) * B * NU2, TWOH = R(2) * H;
    R DPLA_I = R(0), P = R(1), Q = R(1), DR = R(0);
#pragma unroll 1
    for (int it = 0; it < 3; ++it) {
      DPLA_I = DPLA_J;
      const R PLA_I = PLA + DPLA_I;
      DPLA = DPLA_J;
      const R YLD_I = PLA_I == R(0) ? fmin(YMAX, CA) : fmin(YMAX, CA + CB * exp_(CN * log_(PLA_I)));
      DR = R(0.5) * YOUNG * DPLA_I / YLD_I;
      P = R(1) / (R(1) + DR * NU1);
      Q = R(1) / (R(1) + R(3) * DR * NU2);
      const R P2 = P * P, Q2 = Q * Q;
      const R F = A * P2 + B * Q2 - YLD_I * YLD_I;
      const R DF = -(ANU1 * P2 * P + BNU2 * Q2 * Q) * (YOUNG - DR * TWOH) / YLD_I - TWOH * YLD_I;
      DPLA_J = DPLA_I > R(0) ? fmax(R(0), DPLA_I - F / DF) : R(0);
    }
    PLA = PLA + DPLA_I;
    const R T1 = (SN[0] + SN[1]) * P, T2 = (SN[0] - SN[1]) * Q;
    SN[0] = R(0.5) * (T1 + T2);
    SN[1] = R(0.5) * (T1 - T2);
    SN[2] = SN[2] * Q;
    EZZ = DR * T1 / YOUNG;
    return true;
  }
  const R SVM2 = SN[0] * SN[0] + SN[1] * SN[1] - SN[0] * SN[1] + R(3) * SN[2] * SN[2];
  const R YLD2 = YLD * YLD;
  if (!(SVM2 > YLD2 && OFF == R(1))) return false;
  R SVM = ssqrt(SVM2);
  const R H = YLD >= YMAX ? R(0) : CN * CB * exp_((CN - R(1)) * log_(PLA + SMALL));
  const R AA = (SVM2 - YLD2) / (R(5) * SVM2 + R(3) * (-SN[0] * SN[1] + SN[2] * SN[2]));
  const R S1 = (R(1) - R(2) * AA) * SN[0] + AA * SN[1];
  const R S2 = AA * SN[0] + (R(1) - R(2) * AA) * SN[1];
  const R S3 = (R(1) - R(3) * AA) * SN[2];
  SN[0] = S1; SN[1] = S2; SN[2] = S3;
  DPLA = OFF * (SVM - YLD) / (R(3) * G + H);
  PLA = PLA + DPLA;
  YLD = YLD + H * DPLA;
  SVM = ssqrt(SN[0] * SN[0] + SN[1] * SN[1] - SN[0] * SN[1] + R(3) * SN[2] * SN[2]);
  const R RR = fmin(R(1), YLD / fmax(R(EM20), SVM));
  SN[0] *= RR; SN[1] *= RR; SN[2] *= RR;
  EZZ = DPLA * R(0.5) * (SN[0] + SN[1]) / YLD;
  return true;
}

// Element state of one shell, held in registers by the thread that computes it.
// NPT > 0: the integration-point state too (NPT points); NPT = 0: the points'
// state stays in memory and is read and written point by point.
template <class R, int NPT>
struct ShellState {
  static constexpr int NP = NPT > 0 ? NPT : 1;
  R thk, thke, h[3], e[2], jca;
  R sig[NP][5], pla[NP];
  int degen, eid;
};

// IP = false leaves the integration-point stresses and plastic strains out (a caller
// that stages them in shared memory).
template <class R, int NPT, bool IP = true>
__device__ __forceinline__ void shell_load_state(const ShellArgs<R>& a, int e, ShellState<R, NPT>& st) {
  const int nelpad = a.nelpad;
  st.thk = a.thk[e];
  st.thke = a.thke[e];
  st.h[0] = a.hourg[0 * nelpad + e]; st.h[1] = a.hourg[1 * nelpad + e]; st.h[2] = a.hourg[2 * nelpad + e];
  st.e[0] = a.eint[0 * nelpad + e]; st.e[1] = a.eint[1 * nelpad + e];
  st.jca = a.jca ? a.jca[e] : R(0);
  st.degen = a.degen[e];
  st.eid = a.elem_id[e];
  if (NPT > 0 && IP) {
#pragma unroll
    for (int ip = 0; ip < ShellState<R, NPT>::NP; ++ip) {
#pragma unroll
      for (int c = 0; c < 5; ++c) st.sig[ip][c] = a.sig[(ip * 5 + c) * nelpad + e];
      st.pla[ip] = a.pla[ip * nelpad + e];
    }
  }
}

// Writes back the state that shell_element<KEEP = true> kept in registers.
template <class R, int NPT>
__device__ __forceinline__ void shell_store_state(const ShellArgs<R>& a, int e, const ShellState<R, NPT>& st) {
  static_assert(NPT > 0, "kept state needs a fixed number of integration points");
  const int nelpad = a.nelpad;
  a.thk[e] = st.thk;
  a.hourg[0 * nelpad + e] = st.h[0]; a.hourg[1 * nelpad + e] = st.h[1]; a.hourg[2 * nelpad + e] = st.h[2];
  a.eint[0 * nelpad + e] = st.e[0]; a.eint[1 * nelpad + e] = st.e[1];
#pragma unroll
  for (int ip = 0; ip < NPT; ++ip) {
#pragma unroll
    for (int c = 0; c < 5; ++c) a.sig[(ip * 5 + c) * nelpad + e] = st.sig[ip][c];
    a.pla[ip * nelpad + e] = st.pla[ip];
  }
}

// CCOOR3 (from nodal planes in shared memory: x, y, z in FP64 and vx vy vz rx ry rz
// in R, stride NLM, corner k at index lc[k]), CNVEC3, CDERI3, CCOEF3, CDLEN3,
// CDEFO3, CCURV3, CSTRA3, MULAWC (SIGEPS01C / SIGEPS02C -> M2CPLR per
// integration point), CHVIS3, CDT3, CFINT3, the group pressure; corner forces and
// moments out in global axes with CUPDT3P signs.  KEEP = false writes the new
// state to memory at index e, as each quantity is formed; KEEP = true leaves it
// in st (for a caller that keeps the state in registers across cycles).  STAGED
// (with NPT > 0, KEEP false): the old integration-point state is read from shared
// planes, stress component c of point ip at sip[(ip * 5 + c) * sstride] and the
// plastic strain of point ip at sip[(NPT * 5 + ip) * sstride], instead of from st.
template <class R, int NPT, bool KEEP, bool STAGED = false>
__device__ __forceinline__ void shell_element(const ShellArgs<R>& a, const int e, const ShellGroupDesc& gd,
                                              const R DT1, const float* __restrict__ zw, const double* sx,
                                              const double* sy, const double* sz, const R* sv, const int NLM,
                                              const int (&lc)[4], ShellState<R, NPT>& st, R (&Fg)[3][4],
                                              R (&Mg)[3][4], unsigned long long& mykey, unsigned long long& mybits,
                                              double& my_ehou, double& my_wpla, const R* sip = nullptr,
                                              const int sstride = 0) {
  static_assert(!STAGED || (NPT > 0 && !KEEP), "staged state: fixed points, written to memory");
  static_assert(!KEEP || NPT > 0, "kept state needs a fixed number of integration points");
  const int nelpad = a.nelpad;
  const R OFF = R(1);
  // coordinate differences in FP64, cast to R (CNVEC3 / CDERI3 inputs)
  const double x1 = sx[lc[0]], y1 = sy[lc[0]], z1 = sz[lc[0]];
  const R X21 = R(sx[lc[1]] - x1), Y21 = R(sy[lc[1]] - y1), Z21 = R(sz[lc[1]] - z1);
  const R X31 = R(sx[lc[2]] - x1), Y31 = R(sy[lc[2]] - y1), Z31 = R(sz[lc[2]] - z1);
  const R X41 = R(sx[lc[3]] - x1), Y41 = R(sy[lc[3]] - y1), Z41 = R(sz[lc[3]] - z1);
  const R X32 = R(sx[lc[2]] - sx[lc[1]]), Y32 = R(sy[lc[2]] - sy[lc[1]]), Z32 = R(sz[lc[2]] - sz[lc[1]]);
  const R X34 = R(sx[lc[2]] - sx[lc[3]]), Y34 = R(sy[lc[2]] - sy[lc[3]]), Z34 = R(sz[lc[2]] - sz[lc[3]]);
  // ---- CNVEC3, ISHFRAM = 0 (cnvec3.F:66-81) or 2 (cnvec3.F:82-106) ----
  R E1X = X21 + X34, E1Y = Y21 + Y34, E1Z = Z21 + Z34;
  R E2X = X32 + X41, E2Y = Y32 + Y41, E2Z = Z32 + Z41;
  R E3X = E1Y * E2Z - E1Z * E2Y, E3Y = E1Z * E2X - E1X * E2Z, E3Z = E1X * E2Y - E1Y * E2X;
  if (gd.ishfram == 2) {
    R su = E2X * E2X + E2Y * E2Y + E2Z * E2Z;
    E1X = E1X * su + E2Y * E3Z - E2Z * E3Y;
    E1Y = E1Y * su + E2Z * E3X - E2X * E3Z;
    E1Z = E1Z * su + E2X * E3Y - E2Y * E3X;
    su = ssqrt(E1X * E1X + E1Y * E1Y + E1Z * E1Z);
    su = R(1) / (su > R(EM20) ? su : R(EM20));
    E1X *= su; E1Y *= su; E1Z *= su;
    su = ssqrt(E3X * E3X + E3Y * E3Y + E3Z * E3Z);
    su = R(1) / (su > R(EM20) ? su : R(EM20));
    E3X *= su; E3Y *= su; E3Z *= su;
    E2X = E3Y * E1Z - E3Z * E1Y; E2Y = E3Z * E1X - E3X * E1Z; E2Z = E3X * E1Y - E3Y * E1X;
    su = ssqrt(E2X * E2X + E2Y * E2Y + E2Z * E2Z);
    su = R(1) / (su > R(EM20) ? su : R(EM20));
    E2X *= su; E2Y *= su; E2Z *= su;
  } else {
    R su = E3X * E3X + E3Y * E3Y + E3Z * E3Z;
    su = ssqrt(su);
    su = R(1) / (su > R(EM20) ? su : R(EM20));
    E3X *= su; E3Y *= su; E3Z *= su;
    const R q1 = E1X * E1X + E1Y * E1Y + E1Z * E1Z;
    const R q2 = E2X * E2X + E2Y * E2Y + E2Z * E2Z;
    su = ssqrt(q1 / q2);
    E1X = E1X + (E2Y * E3Z - E2Z * E3Y) * su;
    E1Y = E1Y + (E2Z * E3X - E2X * E3Z) * su;
    E1Z = E1Z + (E2X * E3Y - E2Y * E3X) * su;
    su = ssqrt(E1X * E1X + E1Y * E1Y + E1Z * E1Z);
    su = R(1) / (su > R(EM20) ? su : R(EM20));
    E1X *= su; E1Y *= su; E1Z *= su;
    E2X = E3Y * E1Z - E3Z * E1Y; E2Y = E3Z * E1X - E3X * E1Z; E2Z = E3X * E1Y - E3Y * E1X;
  }
  // ---- CDERI3 (cderi3.F:87-190) ----
  const R X2 = E1X * X21 + E1Y * Y21 + E1Z * Z21;
  const R Y2 = E2X * X21 + E2Y * Y21 + E2Z * Z21;
  const R Y3 = E2X * X31 + E2Y * Y31 + E2Z * Z31;
  const R X3 = E1X * X31 + E1Y * Y31 + E1Z * Z31;
  const R X4 = E1X * X41 + E1Y * Y41 + E1Z * Z41;
  const R Y4 = E2X * X41 + E2Y * Y41 + E2Z * Z41;
  R Z2 = E3X * X21 + E3Y * Y21 + E3Z * Z21;      // cderi3.F:108, used by IHBE >= 2
  const R PX1 = R(0.5) * (Y2 - Y4), PY1 = R(0.5) * (X4 - X2), PX2 = R(0.5) * Y3, PY2 = -R(0.5) * X3;
  R AREA = R(2) * (PY2 * PX1 - PY1 * PX2);
  AREA = AREA > R(EM20) ? AREA : R(EM20);
  const R VHX = (-X2 + X3 - X4) / AREA, VHY = (-Y2 + Y3 - Y4) / AREA;
  // ---- CCOEF3 (ccoef3.F:66-160) ----
  const R THK0 = gd.ithk > 0 ? st.thk : st.thke;
  const R VOL0 = THK0 * AREA;
  const R THK02 = THK0 * THK0;
  const R RHO = R(gd.rho0), YM = R(gd.young), NU = R(gd.nu), GG = R(gd.shear);
  const R A11 = R(gd.a11), A12 = R(gd.a12), SSP = R(gd.ssp);
  const R H1 = R(gd.hm), H2 = R(gd.hf), H3 = R(gd.hr);
  const int npt = NPT > 0 ? NPT : gd.npt;
  const R SHF = npt == 1 ? R(0) : R(gd.shf);
  const R GS = GG * SHF;
  // ---- CDLEN3 (cdlen3.F:69-121) ----
  R ALDT;
  {
    const R AL1 = X2 * X2 + Y2 * Y2;
    const R AL2 = (X3 - X2) * (X3 - X2) + (Y3 - Y2) * (Y3 - Y2);
    const R AL6 = X3 * X3 + Y3 * Y3;
    const R AL3 = (X4 - X3) * (X4 - X3) + (Y4 - Y3) * (Y4 - Y3);
    const R AL4 = X4 * X4 + Y4 * Y4;
    const R AL5 = (X4 - X2) * (X4 - X2) + (Y4 - Y2) * (Y4 - Y2);
    R ALMIN = fmin(fmin(AL1, AL2), AL4);
    const R ALQ = fmin(fmin(AL3, AL5), AL6);
    if (AL3 != R(0)) ALMIN = fmin(ALMIN, ALQ);
    R m56 = fmax(AL5, AL6);
    m56 = m56 > R(EM20) ? m56 : R(EM20);
    const R DTDYN = AREA * AREA / m56;
    ALDT = fmax(DTDYN, ALMIN);
    const R DTHOUR = R(0.5) * (ALMIN + ALDT) / fmax(H1, H2);
    if (DTHOUR < ALDT) ALDT = DTHOUR;
    ALDT = ssqrt(ALDT);
  }
  // ---- CDEFO3 (cdefo3.F:84-220): IHBE <= 1, 2 and 4 ----
  R VXl[4], VYl[4], VZl[4], RXl[4], RYl[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const R vx = sv[0 * NLM + lc[k]], vy = sv[1 * NLM + lc[k]], vz = sv[2 * NLM + lc[k]];
    VXl[k] = E1X * vx + E1Y * vy + E1Z * vz;
    VYl[k] = E2X * vx + E2Y * vy + E2Z * vz;
    VZl[k] = E3X * vx + E3Y * vy + E3Z * vz;
    const R rx = sv[3 * NLM + lc[k]], ry = sv[4 * NLM + lc[k]], rz = sv[5 * NLM + lc[k]];
    RXl[k] = E1X * rx + E1Y * ry + E1Z * rz;
    RYl[k] = E2X * rx + E2Y * ry + E2Z * rz;
  }
  // NPT = 5 kernels are launched only when every group is Ishell 1 (IHBE 1) with
  // M2CPLR's radial return (IPLA 0): the other branches compile out of them
  const int IHBE = NPT == 5 ? 1 : gd.ihbe;
  const int IPLA = NPT == 5 ? 0 : gd.ipla;
  R EXX, EYY, EXY, EXZ, EYZ, KXX, KYY, KXY;
  {
    const R VZ13 = VZl[0] - VZl[2], VZ24 = VZl[1] - VZl[3];
    EYZ = PY1 * VZ13 + PY2 * VZ24;
    EXZ = PX1 * VZ13 + PX2 * VZ24;
    R VX13, VX24, VY13, VY24;
    if (IHBE <= 1) {
      Z2 = R(0);
      const R DT1V4 = R(0.25) * DT1;
      const R t2a = PY2 + PY1;
      const R t3a = copysign(fmax(fabs(t2a), R(EM20)), t2a);
      const R t1a = DT1V4 * (VZ13 - VZ24) * (VZ13 - VZ24) / t3a;
      VX13 = VXl[0] - VXl[2] - t1a; VX24 = VXl[1] - VXl[3] + t1a;
      const R t1b = PX2 - PX1;
      const R t3b = copysign(fmax(fabs(t1b), R(EM20)), t1b);
      const R t2b = DT1V4 * (VZ13 + VZ24) * (VZ13 + VZ24) / t3b;
      VY13 = VYl[0] - VYl[2] + t2b; VY24 = VYl[1] - VYl[3] + t2b;
    } else if (IHBE != 4) {
      // IHBE 2 (cdefo3.F:133-172): velocities relative to node 1, warping terms
      const R DT1V4 = R(0.5) * DT1;
      const R GZX = EXZ / AREA, EXZZ2 = GZX * Z2, EXZ2 = GZX * GZX * DT1V4;
      VXl[2] = VXl[2] - EXZ2 * X3 - VXl[0];
      VXl[1] = VXl[1] + EXZZ2 - EXZ2 * X2 - VXl[0];
      VXl[3] = VXl[3] + EXZZ2 - EXZ2 * X4 - VXl[0];
      VXl[0] = R(0);
      const R GZY = EYZ / AREA, EYZZ2 = GZY * Z2, EYZ2 = GZY * GZY * DT1V4;
      VYl[2] = VYl[2] - EYZ2 * Y3 - VYl[0];
      VYl[1] = VYl[1] + EYZZ2 - EYZ2 * Y2 - VYl[0];
      VYl[3] = VYl[3] + EYZZ2 - EYZ2 * Y4 - VYl[0];
      VYl[0] = R(0);
      const R ZZZ = (EXZ2 + EYZ2) * Z2;
      VZl[2] = VZl[2] - GZY * Y3 - GZX * X3 - VZl[0];
      VZl[1] = VZl[1] - GZY * Y2 - GZX * X2 - ZZZ - VZl[0];
      VZl[3] = VZl[3] - GZY * Y4 - GZX * X4 - ZZZ - VZl[0];
      VZl[0] = R(0);
      VX13 = -VXl[2]; VX24 = VXl[1] - VXl[3];
      VY13 = -VYl[2]; VY24 = VYl[1] - VYl[3];
    } else {
      // IHBE 4 (cdefo3.F:174-216): z1 = z3 = 0, z4 = z2
      const R DT1V4 = R(0.5) * DT1, ZZ2 = R(0.5) * Z2;
      const R GZX = EXZ / AREA, EXZZ2 = GZX * ZZ2, EXZ2 = GZX * GZX * DT1V4;
      const R EXZ2PY2 = EXZ2 * PY2, EXZ2PY1 = EXZ2 * PY1;
      VXl[0] = VXl[0] - EXZZ2 - EXZ2PY2;
      VXl[2] = VXl[2] - EXZZ2 + EXZ2PY2;
      VXl[1] = VXl[1] + EXZZ2 + EXZ2PY1;
      VXl[3] = VXl[3] + EXZZ2 - EXZ2PY1;
      const R GZY = EYZ / AREA, EYZZ2 = GZY * ZZ2, EYZ2 = GZY * GZY * DT1V4;
      const R EYZ2PX2 = EYZ2 * PX2, EYZ2PX1 = EYZ2 * PX1;
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
    // ---- CCURV3 (ccurv3.F:61-86) ----
    const R RX13 = RXl[0] - RXl[2], RXAV = RXl[0] + RXl[1] + RXl[2] + RXl[3], RX24 = RXl[1] - RXl[3];
    KYY = -PY1 * RX13 - PY2 * RX24;
    R kxy = PX1 * RX13 + PX2 * RX24;
    const R RY13 = RYl[0] - RYl[2], RYAV = RYl[0] + RYl[1] + RYl[2] + RYl[3], RY24 = RYl[1] - RYl[3];
    KXX = PX1 * RY13 + PX2 * RY24;
    KXY = PY1 * RY13 + PY2 * RY24 - kxy;
    EXZ = EXZ + RYAV * (R(0.25) * AREA);
    EYZ = EYZ - RXAV * (R(0.25) * AREA);
    // ---- CSTRA3 (cstra3.F:91-101) ----
    const R FAC1 = DT1 / AREA;
    EXX *= FAC1; EYY *= FAC1; EXY *= FAC1; EYZ *= FAC1; EXZ *= FAC1;
    KXX *= FAC1; KYY *= FAC1; KXY *= FAC1;
  }
  // ---- MULAWC layer loop (mulawc.F90:530-560, 596-1100, 2603-2620, 2930-2990) ----
  const float* Z0 = zw + (npt - 1) * 33;      // [Z0 | WF | WM] of the npt-point rule
  const float* WF = Z0 + 11;
  const float* WM = Z0 + 22;
  R FOR[5] = {R(0), R(0), R(0), R(0), R(0)}, MOM[3] = {R(0), R(0), R(0)};
  R FOLD[5] = {R(0), R(0), R(0), R(0), R(0)}, MOLD[3] = {R(0), R(0), R(0)};
  R THKN = st.thk;
  const R CA = gd.has_jca ? st.jca : R(gd.jc_a);
  const R CB = R(gd.jc_b), CN = R(gd.jc_n), YMAX = R(gd.sigmax);
  double wpla = 0.0;
  // SIGY for CHSTI3: EP30 (ccoor3.F:126); LAW2 adds each point's yield / NPTT
  // (mulawc.F90:565, sigeps02c.F:186-188)
  R SIGY = gd.law == 1 ? R(1e30) : R(0);
#pragma unroll
  for (int ip = 0; ip < (NPT > 0 ? NPT : 10); ++ip) {
    if (NPT == 0 && ip >= npt) break;
    const R wf = R(NPT == 5 ? coq5(1, ip) : WF[ip]), wm = R(NPT == 5 ? coq5(2, ip) : WM[ip]);
    R SO[5], SN[5];
    if (STAGED) {
#pragma unroll
      for (int c = 0; c < 5; ++c) SO[c] = sip[(ip * 5 + c) * sstride];
    } else if (NPT > 0) {
#pragma unroll
      for (int c = 0; c < 5; ++c) SO[c] = st.sig[NPT > 0 ? ip : 0][c];
    } else {
#pragma unroll
      for (int c = 0; c < 5; ++c) SO[c] = a.sig[(ip * 5 + c) * nelpad + e];
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) FOLD[c] = FOLD[c] + wf * SO[c];
#pragma unroll
    for (int c = 0; c < 3; ++c) MOLD[c] = MOLD[c] + wm * SO[c];
    const R THKLYL = wf * THK0;
    const R ZT = R(NPT == 5 ? coq5(0, ip) : Z0[ip]) * THK0;
    const R DXX = EXX + ZT * KXX, DYY = EYY + ZT * KYY, DXY = EXY + ZT * KXY;
    R EZZ = R(0);
    if (gd.law == 1) {
      // SIGEPS01C (sigeps01c.F:130-146)
      SN[0] = SO[0] + A11 * DXX + A12 * DYY;
      SN[1] = SO[1] + A12 * DXX + A11 * DYY;
      SN[2] = SO[2] + GG * DXY;
      SN[3] = SO[3] + GS * EYZ;
      SN[4] = SO[4] + GS * EXZ;
      EZZ = -NU * (DXX + DYY) / (R(1) - NU);
    } else {
      // SIGEPS02C -> M2CPLR, IPLA = 0 radial return (m2cplr.F:96-230)
      const R A1 = YM / (R(1) - NU * NU), A2 = A1 * NU;
      SN[0] = SO[0] + A1 * DXX + A2 * DYY;
      SN[1] = SO[1] + A2 * DXX + A1 * DYY;
      SN[2] = SO[2] + GG * DXY;
      SN[3] = SO[3] + GS * EYZ;
      SN[4] = SO[4] + GS * EXZ;
      R PLA = STAGED ? sip[((NPT > 0 ? NPT : 1) * 5 + ip) * sstride]
              : NPT > 0 ? st.pla[NPT > 0 ? ip : 0] : a.pla[ip * nelpad + e];
      R YLD = PLA == R(0) ? CA : CA + CB * exp_(CN * log_(PLA));
      YLD = fmin(YLD, YMAX);
      R DPLA = R(0);
      if (IPLA == 0) {
        const R SVM = ssqrt(SN[0] * SN[0] + SN[1] * SN[1] - SN[0] * SN[1] + R(3) * SN[2] * SN[2]);
        const R RR = fmin(R(1), YLD / (SVM + R(EM15)));
        if (RR < R(1)) {
          SN[0] *= RR; SN[1] *= RR; SN[2] *= RR;
          DPLA = OFF * fmax(R(0), (SVM - YLD) / YM);
          EZZ = DPLA * (R(0.5) * (SN[0] + SN[1])) / YLD;
          PLA = PLA + DPLA;
          if (KEEP) st.pla[NPT > 0 ? ip : 0] = PLA;
          else a.pla[ip * nelpad + e] = PLA;
        }
      } else {
        if (m2cplr_iterative<R>(IPLA, SN, PLA, YLD, DPLA, EZZ, CA, CB, CN, YMAX, YM, NU, GG, OFF)) {
          if (KEEP) st.pla[NPT > 0 ? ip : 0] = PLA;
          else a.pla[ip * nelpad + e] = PLA;
        }
      }
      SIGY = SIGY + YLD / R(npt);
      EZZ = -(DXX + DYY) * NU - (R(1) - R(2) * NU) * EZZ;   // sigeps02c.F:215-224
      EZZ = EZZ / (R(1) - NU);
      if (DPLA != R(0)) wpla += (double)YLD * (double)DPLA * (double)AREA * (double)THKLYL;
    }
    THKN = THKN + EZZ * THKLYL * OFF;
    if (KEEP) {
#pragma unroll
      for (int c = 0; c < 5; ++c) st.sig[NPT > 0 ? ip : 0][c] = SN[c];
    } else {
#pragma unroll
      for (int c = 0; c < 5; ++c) a.sig[(ip * 5 + c) * nelpad + e] = SN[c];
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) FOR[c] = FOR[c] + wf * SN[c];
#pragma unroll
    for (int c = 0; c < 3; ++c) MOM[c] = MOM[c] + wm * SN[c];
  }
  my_wpla = wpla;
  if (KEEP) st.thk = THKN > R(EM30) ? THKN : R(EM30);
  else a.thk[e] = THKN > R(EM30) ? THKN : R(EM30);
  {
    const R DEGMB = FOLD[0] * EXX + FOLD[1] * EYY + FOLD[2] * EXY + FOLD[3] * EYZ + FOLD[4] * EXZ +
                    (FOR[0] * EXX + FOR[1] * EYY + FOR[2] * EXY + FOR[3] * EYZ + FOR[4] * EXZ);
    const R DEGFX = MOLD[0] * KXX + MOLD[1] * KYY + MOLD[2] * KXY +
                    (MOM[0] * KXX + MOM[1] * KYY + MOM[2] * KXY);
    const R VOL2 = R(0.5) * VOL0;
    if (KEEP) {
      st.e[0] = st.e[0] + DEGMB * VOL2;
      st.e[1] = st.e[1] + DEGFX * THK0 * VOL2;
    } else {
      a.eint[0 * nelpad + e] = st.e[0] + DEGMB * VOL2;
      a.eint[1 * nelpad + e] = st.e[1] + DEGFX * THK0 * VOL2;
    }
  }
  // ---- hourglass forces (cforc3.F:593-640): MHVIS3 for one integration point,
  // CHSTI3 for IHBE = 2, CHVIS3 otherwise; ISMSTR = 2, HELAS = HVISC = 1/2, HVLIN = 0.
  // H1j/H2j/H3j: membrane x, y and bending forces of corners 1..3 (corner 4 from
  // the zero sum), HOUR4/HOUR5 the hourglass moments ----
  R H1j[3], H2j[3], H3j[3], HOUR4 = R(0), HOUR5 = R(0);
  {
    R GAMA[4];
    if (IHBE >= 1) {
      const R px1v = PX1 * VHX, px2v = PX2 * VHX, py1v = PY1 * VHY, py2v = PY2 * VHY;
      GAMA[0] = OFF * (R(1) - px1v - py1v);
      GAMA[2] = OFF * (R(1) + px1v + py1v);
      GAMA[1] = OFF * (-R(1) - px2v - py2v);
      GAMA[3] = OFF * (-R(1) + px2v + py2v);
    } else {
      GAMA[0] = OFF; GAMA[2] = OFF; GAMA[1] = -OFF; GAMA[3] = -OFF;
    }
    R hour1, hour2, hour3, EHOU;
    if (npt == 1) {
      // MHVIS3 (mhvis3.F:109-363): elastic terms only, V-shape bending damping Dn,
      // no hourglass moments; IHBE >= 1 here (one point turns Ishell 2 into 1)
      const R H4 = R(gd.dn);
      R H4L = R(0.25) * RHO * THK0 * ssqrt(R(0.5) * H4 * AREA);
      R H4Q = ssqrt(R(0.5) * H4) * H4L * R(100);
      H4L = H4L * SSP;
      const R FAC = R(0.25) * YM * THK0 * DT1 * R(0.5);
      R H1e = H1 * FAC, H2e = H2 * FAC;
      if (st.degen) { H4L = H4Q = H1e = H2e = R(0); }
      const R HG1 = VXl[0] * GAMA[0] + VXl[1] * GAMA[1] + VXl[2] * GAMA[2] + VXl[3] * GAMA[3];
      const R HG2 = VYl[0] * GAMA[0] + VYl[1] * GAMA[1] + VYl[2] * GAMA[2] + VYl[3] * GAMA[3];
      hour1 = st.h[0] + HG1 * H1e;
      hour2 = st.h[1] + HG2 * H1e;
      // the viscous factors H1L, H1Q, H2L, H2Q of MHVIS3 are zero: (HOUR + 0) * GAMA
      R Hm1[4], Hm2[4], Hb[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) { Hm1[k] = hour1 * GAMA[k]; Hm2[k] = hour2 * GAMA[k]; }
      EHOU = VXl[0] * Hm1[0] + VXl[1] * Hm1[1] + VXl[2] * Hm1[2] + VXl[3] * Hm1[3] +
             VYl[0] * Hm2[0] + VYl[1] * Hm2[1] + VYl[2] * Hm2[2] + VYl[3] * Hm2[3];
      R HGb = VZl[0] * GAMA[0] + VZl[1] * GAMA[1] + VZl[2] * GAMA[2] + VZl[3] * GAMA[3];
      hour3 = st.h[2] + HGb * H2e;
#pragma unroll
      for (int k = 0; k < 4; ++k) Hb[k] = hour3 * GAMA[k];
      HGb = VZl[0] + VZl[1] - VZl[2] - VZl[3];
      HGb = HGb * (H4L + H4Q * fabs(HGb));
      Hb[0] = Hb[0] + HGb; Hb[1] = Hb[1] + HGb; Hb[2] = Hb[2] - HGb; Hb[3] = Hb[3] - HGb;
      HGb = VZl[0] - VZl[1] - VZl[2] + VZl[3];
      HGb = HGb * (H4L + H4Q * fabs(HGb));
      Hb[0] = Hb[0] + HGb; Hb[1] = Hb[1] - HGb; Hb[2] = Hb[2] - HGb; Hb[3] = Hb[3] + HGb;
#pragma unroll
      for (int k = 0; k < 3; ++k) { H1j[k] = Hm1[k]; H2j[k] = Hm2[k]; H3j[k] = Hb[k]; }
      EHOU = EHOU + VZl[0] * Hb[0] + VZl[1] * Hb[1] + VZl[2] * Hb[2] + VZl[3] * Hb[3];
      my_ehou = (double)(DT1 * EHOU);
    } else if (IHBE == 2) {
      // CHSTI3 (chsti3.F:119-320): elastic stiffness bounded by the yield stress,
      // viscous rotational terms with SRH3 = sqrt(hr) (resol_init.F:676-682)
      const R H3s = R(sqrt(gd.hr));
      const R SHFPR3 = SHF / (R(3) * (R(1) + NU));
      R H3L = H3s * R(0.072169) * (R(0.25) * RHO * THK02) * AREA;
      R H3Q = H3s * H3L * R(100);
      H3L = H3L * SSP;
      const R FAC = YM * THK0 * DT1 * R(0.125);
      R H1e = H1 * FAC;
      const R B1 = PX1 * PX1 + PY1 * PY1, B2 = PX2 * PX2 + PY2 * PY2;
      R H2e = H2 * FAC * THK02 * SHFPR3 / (B1 + B2);
      if (st.degen) { H3Q = H3L = H1e = H2e = R(0); }
      R HG1 = VXl[0] * GAMA[0] + VXl[1] * GAMA[1] + VXl[2] * GAMA[2] + VXl[3] * GAMA[3];
      R HG2 = VYl[0] * GAMA[0] + VYl[1] * GAMA[1] + VYl[2] * GAMA[2] + VYl[3] * GAMA[3];
      hour1 = st.h[0] + HG1 * H1e;
      hour2 = st.h[1] + HG2 * H1e;
      R FMAX = R(0.5) * SIGY * THK0 * ssqrt(AREA) * H1;
      hour1 = copysign(fmin(fabs(hour1), FMAX), hour1);
      hour2 = copysign(fmin(fabs(hour2), FMAX), hour2);
#pragma unroll
      for (int k = 0; k < 3; ++k) { H1j[k] = hour1 * GAMA[k]; H2j[k] = hour2 * GAMA[k]; }
      EHOU = hour1 * HG1 + hour2 * HG2;
      HG1 = VZl[0] * GAMA[0] + VZl[1] * GAMA[1] + VZl[2] * GAMA[2] + VZl[3] * GAMA[3];
      hour3 = st.h[2] + HG1 * H2e;
      FMAX = R(0.25) * SIGY * THK0 * THK0 * H2;
      hour3 = copysign(fmin(fabs(hour3), FMAX), hour3);
#pragma unroll
      for (int k = 0; k < 3; ++k) H3j[k] = hour3 * GAMA[k];
      EHOU = EHOU + hour3 * HG1;
      HG1 = RXl[0] - RXl[1] + RXl[2] - RXl[3];
      HG2 = RYl[0] - RYl[1] + RYl[2] - RYl[3];
      HOUR4 = HG1 * (H3L + H3Q * fabs(HG1));
      HOUR5 = HG2 * (H3L + H3Q * fabs(HG2));
      EHOU = EHOU + HOUR4 * HG1 + HOUR5 * HG2;
      my_ehou = (double)(DT1 * EHOU * OFF);
    } else {
      // CHVIS3 (chvis3.F:116-300)
      const R SHFPR3 = SHF / (R(3) * (R(1) + NU));
      const R R1 = R(0.25) * RHO * R(100);
      const R A1c = R1 * (R(0.5) * H1);
      const R A3c = R1 * (R(0.5) * H2) * ssqrt(SHFPR3);
      const R A5c = R(0.5) * H3 * R1 * R(0.072169);
      const R R0e = R(0.25) * YM * R(0.5);
      const R A7c = H1 * R0e, A8c = H2 * R0e * SHFPR3;
      const R T2A = THK02 * AREA;
      R H1Q = A1c * ssqrt(T2A), H2Q = A3c * THK02, H3Q = A5c * T2A;
      const R TD = THK0 * DT1;
      R HH1 = A7c * TD;
      const R B1 = PX1 * PX1 + PY1 * PY1, B2 = PX2 * PX2 + PY2 * PY2;
      R HH2 = A8c * THK02 * TD / (B1 + B2);
      if (st.degen) { H1Q = H2Q = H3Q = HH1 = HH2 = R(0); }
      R HG1, HG2;
      if (IHBE < 1) {
        HG1 = (VXl[0] - VXl[1] + VXl[2] - VXl[3]) * OFF;
        HG2 = (VYl[0] - VYl[1] + VYl[2] - VYl[3]) * OFF;
      } else {
        HG1 = VXl[0] * GAMA[0] + VXl[1] * GAMA[1] + VXl[2] * GAMA[2] + VXl[3] * GAMA[3];
        HG2 = VYl[0] * GAMA[0] + VYl[1] * GAMA[1] + VYl[2] * GAMA[2] + VYl[3] * GAMA[3];
      }
      hour1 = st.h[0] + HG1 * HH1;
      hour2 = st.h[1] + HG2 * HH1;
      const R HOUR1A = hour1 + HG1 * (H1Q * fabs(HG1));
      const R HOUR2A = hour2 + HG2 * (H1Q * fabs(HG2));
#pragma unroll
      for (int k = 0; k < 3; ++k) { H1j[k] = HOUR1A * GAMA[k]; H2j[k] = HOUR2A * GAMA[k]; }
      EHOU = HOUR1A * HG1 + HOUR2A * HG2;
      if (IHBE < 1) HG1 = (VZl[0] - VZl[1] + VZl[2] - VZl[3]) * OFF;
      else HG1 = VZl[0] * GAMA[0] + VZl[1] * GAMA[1] + VZl[2] * GAMA[2] + VZl[3] * GAMA[3];
      hour3 = st.h[2] + HG1 * HH2;
      const R HOUR3A = hour3 + HG1 * (H2Q * fabs(HG1));
#pragma unroll
      for (int k = 0; k < 3; ++k) H3j[k] = HOUR3A * GAMA[k];
      EHOU = EHOU + HOUR3A * HG1;
      HG1 = RXl[0] - RXl[1] + RXl[2] - RXl[3];
      HG2 = RYl[0] - RYl[1] + RYl[2] - RYl[3];
      HOUR4 = HG1 * (H3Q * fabs(HG1));
      HOUR5 = HG2 * (H3Q * fabs(HG2));
      EHOU = EHOU + HOUR4 * HG1 + HOUR5 * HG2;
      my_ehou = (double)(DT1 * EHOU * OFF);
    }
    if (KEEP) { st.h[0] = hour1; st.h[1] = hour2; st.h[2] = hour3; }
    else { a.hourg[0 * nelpad + e] = hour1; a.hourg[1 * nelpad + e] = hour2; a.hourg[2 * nelpad + e] = hour3; }
  }
  // ---- CDT3 (cdt3.F:110-115, 203-214) ----
  {
    const R DT = R(gd.dtfac) * ALDT / SSP;
    if ((double)DT <= gd.dtmin) raise_error(a.err, 5, st.eid);
    mykey = dt_key((double)DT, 3, st.eid);
    mybits = (unsigned long long)__double_as_longlong((double)DT);
  }
  // ---- CFINT3, ISIGI = 0 (cfint3.F:173-260) ----
  {
    const R F1A = FOR[0] * THK0, F2A = FOR[1] * THK0, F3A = FOR[2] * THK0, F4A = FOR[3] * THK0, F5A = FOR[4] * THK0;
    R M4 = F4A * AREA, M5 = F5A * AREA;
    if (IHBE >= 2 && npt != 1) {            // cfint3.F:208-214, warping moments
      M4 = M4 + (H2j[0] + H2j[2]) * Z2;
      M5 = M5 + (H1j[0] + H1j[2]) * Z2;
    }
    M4 = M4 * R(0.25); M5 = M5 * R(0.25);
    const R F12 = F1A * PX2 + F3A * PY2, F22 = F2A * PY2 + F3A * PX2, F32 = F5A * PX2 + F4A * PY2;
    const R F11 = F1A * PX1 + F3A * PY1, F21 = F2A * PY1 + F3A * PX1, F31 = F5A * PX1 + F4A * PY1;
    const R Gc[3][3] = {{F11 + H1j[0], F12 + H1j[1], H1j[2] - F11},
                        {F21 + H2j[0], F22 + H2j[1], H2j[2] - F21},
                        {F31 + H3j[0], F32 + H3j[1], H3j[2] - F31}};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      Fg[0][k] = E1X * Gc[0][k] + E2X * Gc[1][k] + E3X * Gc[2][k];
      Fg[1][k] = E1Y * Gc[0][k] + E2Y * Gc[1][k] + E3Y * Gc[2][k];
      Fg[2][k] = E1Z * Gc[0][k] + E2Z * Gc[1][k] + E3Z * Gc[2][k];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) Fg[c][3] = -Fg[c][0] - Fg[c][1] - Fg[c][2];
    const R M1A = MOM[0] * THK02, M2A = MOM[1] * THK02, M3A = MOM[2] * THK02;
    const R M11 = -M2A * PY1 - M3A * PX1, M21 = M1A * PX1 + M3A * PY1;
    const R M12 = -M2A * PY2 - M3A * PX2, M22 = M1A * PX2 + M3A * PY2;
    const R G1m[4] = {M11 - M4 + HOUR4 * OFF, M12 - M4 - HOUR4 * OFF, -M11 - M4 + HOUR4 * OFF, -M12 - M4 - HOUR4 * OFF};
    const R G2m[4] = {M21 + M5 + HOUR5 * OFF, M22 + M5 - HOUR5 * OFF, -M21 + M5 + HOUR5 * OFF, -M22 + M5 - HOUR5 * OFF};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      Mg[0][k] = E1X * G1m[k] + E2X * G2m[k];
      Mg[1][k] = E1Y * G1m[k] + E2Y * G2m[k];
      Mg[2][k] = E1Z * G1m[k] + E2Z * G2m[k];
    }
  }
  // ---- uniform pressure (load_pressure.F:201-207): F = -p N / 8, N = x13 x x24,
  // the diagonals taken in FP64 and the cross product in R ----
  R PF[3] = {R(0), R(0), R(0)};
  if (gd.pressure != 0.0) {
    const R ax = R(sx[lc[2]] - x1), ay = R(sy[lc[2]] - y1), az = R(sz[lc[2]] - z1);
    const R bx = R(sx[lc[3]] - sx[lc[1]]), by = R(sy[lc[3]] - sy[lc[1]]), bz = R(sz[lc[3]] - sz[lc[1]]);
    const R NX = ay * bz - az * by, NY = az * bx - ax * bz, NZ = ax * by - ay * bx;
    const R AA = -R(gd.pressure) * R(0.125);
    PF[0] = AA * NX; PF[1] = AA * NY; PF[2] = AA * NZ;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    Fg[0][k] = -Fg[0][k] + PF[0]; Fg[1][k] = -Fg[1][k] + PF[1]; Fg[2][k] = -Fg[2][k] + PF[2];
    Mg[0][k] = -Mg[0][k]; Mg[1][k] = -Mg[1][k]; Mg[2][k] = -Mg[2][k];
  }
}

// Shared planes of staged integration-point state of the NPT-point shell patch
// kernel: 5 stresses and the plastic strain per point (none for the generic kernel).
__host__ __device__ constexpr int shell_staged_planes(int npt) { return npt > 0 ? 6 * npt : 0; }

// ===========================================================================
// shell patch kernel
// ===========================================================================
// Per element (thread): CCOOR3, CNVEC3, CDERI3, CCOEF3, CDLEN3, CDEFO3, CCURV3,
// CSTRA3, MULAWC (SIGEPS01C / SIGEPS02C -> M2CPLR per integration point),
// CHVIS3, CDT3, CFINT3; forces and moments into shared memory (CUPDT3P signs).
// NPT > 0: every group of the launch has NPT integration points; their state is
// loaded up front into registers, or with STG staged in shared memory by bulk
// copies and read point by point; NPT = 0: generic 1..10 points, read from global
// memory in the layer loop.
template <class R, int TILE, int NPT, bool STG>
__global__ void __launch_bounds__(TILE, min_blocks(STG ? Occupancy<R>::shell_staged : Occupancy<R>::shell, TILE))
shell_patch_kernel(ShellArgs<R> a, int parity, const float* __restrict__ zw) {
  typedef typename Vec4<R>::T R4;
  // NPT > 0: the patch's integration-point stresses and plastic strains are staged in
  // NSP shared planes of TILE by bulk copies, read point by point in the layer loop
  constexpr int NSP = STG ? shell_staged_planes(NPT) : 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned long long s_key[TILE / 32], s_bits[TILE / 32];
  __shared__ double s_s0[TILE / 32], s_s1[TILE / 32];
  __shared__ __align__(8) unsigned long long s_bar;
  const int p = blockIdx.x;
  const int tid = threadIdx.x;
  // element index and node-list slots follow from (p, tid) alone (patches padded
  // to TILE elements and nlmax nodes): loads start before the descriptors arrive
  const int NLM = a.nlmax;
  const int e = p * TILE + tid;
  const PatchInfo pi = a.patch[p];
  // issued now, used at the end: the patch's slot numbers (up to two per thread)
  // and its cumulative energy partials
  const int slot0 = tid < NLM ? a.patch_slots[p * NLM + tid] : -1;
  const int slot1 = tid + TILE < NLM ? a.patch_slots[p * NLM + tid + TILE] : -1;
  double pre_ehour = 0.0, pre_wpla = 0.0;
  if (tid == 0) { pre_ehour = a.blk_ehour[p]; pre_wpla = a.blk_wpla[p]; }
  R* sip = reinterpret_cast<R*>(smem_raw);
  double* sx = reinterpret_cast<double*>(sip + NSP * TILE);
  double* sy = sx + NLM;
  double* sz = sy + NLM;
  R* sv = reinterpret_cast<R*>(sz + NLM);   // vx vy vz rx ry rz: 6 planes of NLM
  R* sc = sv + 6 * NLM;                     // 24 planes of TILE: component c of corner k at (c*4+k)
  unsigned short* sinc = reinterpret_cast<unsigned short*>(sc + 24 * TILE);
  const int nelpad = a.nelpad;
  // per-element loads issued before the staging barrier (overlap with the gathers)
  // padding elements (tid >= nel) hold valid state: load unconditionally
  if (NSP > 0 && tid == 0) {   // written two launches back: issued before the wait
    mbar_init(&s_bar);
    const unsigned pl = TILE * sizeof(R);
    const size_t e0 = (size_t)p * TILE;
    mbar_expect_tx(&s_bar, NSP * pl);
#pragma unroll 1
    for (int q = 0; q < 5 * NPT; ++q) bulk_g2s(sip + q * TILE, a.sig + (size_t)q * nelpad + e0, pl, &s_bar);
#pragma unroll 1
    for (int ip = 0; ip < NPT; ++ip)
      bulk_g2s(sip + (5 * NPT + ip) * TILE, a.pla + (size_t)ip * nelpad + e0, pl, &s_bar);
  }
  const uint2 cw = a.conn[e];
  ShellState<R, NPT> st;
  shell_load_state<R, NPT, NSP == 0>(a, e, st);
  {
    const unsigned* src = reinterpret_cast<const unsigned*>(a.inc + (size_t)p * a.inc_stride);
    unsigned* dst = reinterpret_cast<unsigned*>(sinc);
    for (int i = tid; i < a.inc_stride / 2; i += TILE) dst[i] = src[i];
  }
  // the patch's node numbers (static) go to the corner-force planes before the
  // wait, each entry read back by the thread that wrote it; X, V, VR and the cycle's
  // time come from the previous node pass
  int* sidx = reinterpret_cast<int*>(sc);   // NLM <= 4 * TILE entries
  for (int j = tid; j < NLM; j += TILE) sidx[j] = a.patch_nodes[p * NLM + j];
  pdl_wait();
  pdl_trigger();
  for (int j = tid; j < NLM; j += TILE) {
    const int g = sidx[j];
    const double4 xx = a.X[g];
    const R4 vv = a.V[g];
    const R4 rr = a.VR[g];
    sx[j] = xx.x; sy[j] = xx.y; sz[j] = xx.z;
    sv[0 * NLM + j] = vv.x; sv[1 * NLM + j] = vv.y; sv[2 * NLM + j] = vv.z;
    sv[3 * NLM + j] = rr.x; sv[4 * NLM + j] = rr.y; sv[5 * NLM + j] = rr.z;
  }
  const ShellGroupDesc gd = a.groups[pi.group];
  const bool active = tid < pi.nel;
  const int nl = pi.nloc;
  const PartTime& tm = a.time[parity * a.nparts + pi.part];
  const R DT1 = R(tm.dt2);
  __syncthreads();
  if (NSP > 0 && !mbar_wait0(&s_bar, STAGE_WAIT_TRIES)) raise_error(a.err, 7, p);

  int lc[4];
  int color = -1;
  R Fg[3][4], Mg[3][4];
  unsigned long long mykey = ~0ull, mybits = ~0ull;
  double my_ehou = 0.0, my_wpla = 0.0;
  if (active) {
    lc[0] = cw.x & 0xffffu; lc[1] = cw.x >> 16; lc[2] = cw.y & 0xffffu; lc[3] = cw.y >> 16;
    color = lc[0] >> COLOR_SHIFT;
    lc[0] &= LOCAL_MASK;
    shell_element<R, NPT, false, (NSP > 0)>(a, e, gd, DT1, zw, sx, sy, sz, sv, NLM, lc, st, Fg, Mg, mykey, mybits,
                                            my_ehou, my_wpla, sip + tid, TILE);
  }
  // ---- patch assembly: corner forces and moments to shared memory, then each patch
  // node sums its incident corners in ascending (element, corner) order ----
  if (active) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sc[(c * 4 + k) * TILE + tid] = Fg[c][k];
        sc[((c + 3) * 4 + k) * TILE + tid] = Mg[c][k];
      }
    }
  }
  (void)color;
  __syncthreads();
  for (int j = tid; j < nl; j += TILE) {
    R f0 = R(0), f1 = R(0), f2 = R(0), m0 = R(0), m1 = R(0), m2 = R(0);
    const int i1 = sinc[j + 1];
    for (int i = sinc[j]; i < i1; ++i) {
      const int o = sinc[NLM + 1 + i];     // corner k of element t: k * TILE + t
      f0 += sc[o]; f1 += sc[4 * TILE + o]; f2 += sc[8 * TILE + o];
      m0 += sc[12 * TILE + o]; m1 += sc[16 * TILE + o]; m2 += sc[20 * TILE + o];
    }
    const int s = j == tid ? slot0 : j == tid + TILE ? slot1 : a.patch_slots[p * NLM + j];
    a.fslot[s] = mk4(f0, f1, f2, R(0));
    a.mslot[s] = mk4(m0, m1, m2, R(0));
  }
  block_reduce<TILE>(mykey, mybits, my_ehou, my_wpla, s_key, s_bits, s_s0, s_s1);
  if (tid == 0) {
    PartAcc* acc = &a.acc[parity * a.nparts + pi.part];
    atomicMin(&acc->dtkey, mykey);
    atomicMin(&acc->dtbits, mybits);
    a.blk_ehour[p] = pre_ehour + my_ehou;
    a.blk_wpla[p] = pre_wpla + my_wpla;
  }
}

// ===========================================================================
// node kernel: ASSPAR4 + dt (resol.F:5853-6226) + ACCELE + BCS10 + VELOCITY + DEPLA
// ===========================================================================
// dt logic (resol.F:5853-5858, 6080, 6224-6226) of one part: DT2 from the
// cycle's element reduction, the growth cap and DTMX, and the element that set it
__device__ __forceinline__ void cycle_dt(const PartAcc& ac, const PartTime& t0, const double growth, const double dtmx,
                                         const int split, double& DT2, int& ityp, int& nelt) {
  const double dt2t = __longlong_as_double((long long)ac.dtbits);
  DT2 = 1e6;                                         // EP06
  ityp = t0.ityptst;
  nelt = t0.neltst;
  if (ac.dtbits != ~0ull && dt2t < DT2) {
    DT2 = dt2t;
    ityp = (ac.dtkey & 0x80000000ull) ? 1 : 3;
    nelt = (int)(ac.dtkey & 0x7fffffffull);
  }
  const double cap = growth * t0.dt2old;
  DT2 = DT2 < cap ? DT2 : cap;
  DT2 = DT2 < dtmx ? DT2 : dtmx;
  if (split) DT2 = (double)(float)DT2;
}

// ACCELE, BCS10 (global axes or a skew frame, bcs1.F), the rigid-link mean
// (RLINK10, then BCS10 again), the kinetic energy at mid-step, VELOCITY and DEPLA
// (FP64 accumulation) of one node, translations and (rot) rotations, from its
// summed force (ax, ay, az) and moment (rx, ry, rz).  Shared by the node pass and
// the persistent kernel, so that both produce the same bits.  want_ek = false
// skips the kinetic energies (a cycle whose energies nobody reads).
template <class R>
__device__ __forceinline__ void node_update(const NodeArgs<R>& a, const int n, const unsigned char code, const bool rot,
                                            R ax, R ay, R az, R rx, R ry, R rz, const R ms, const double DT1,
                                            const double DT2, const double DT12, double& px, double& py, double& pz,
                                            double& qx, double& qy, double& qz, typename Vec4<R>::T& v,
                                            typename Vec4<R>::T& w, double& ek, double& ekr, const bool want_ek = true) {
  // ACCELE (accele.F:63-80)
  if (ms > R(0)) { const R r = R(1) / ms; ax *= r; ay *= r; az *= r; }
  else { ax = ay = az = R(0); }
  if (!isfinite((double)ax + (double)ay + (double)az)) raise_error(a.err, 6, n);
  // BCS10 (bcs1.F:52-100)
  const R* sk = (code & 128) ? a.skews + 9 * a.skew_of[n] : nullptr;
  if (sk) {
    bcs1v_skew(code & 7, sk, v.x, v.y, v.z);
    bcs1v_skew(code & 7, sk, ax, ay, az);
  } else {
    if (code & 4) { v.x = R(0); ax = R(0); }
    if (code & 2) { v.y = R(0); ay = R(0); }
    if (code & 1) { v.z = R(0); az = R(0); }
  }
  if (code & 64) {      // RLINK10 (resol.F:7053), then BCS10 again (resol.F:7458)
    const LinkMean* lm = &a.link_mean[a.link_of[n]];
    const int ic = lm->ic;
    if (ic & 4) ax = R(lm->a[0]);
    if (ic & 2) ay = R(lm->a[1]);
    if (ic & 1) az = R(lm->a[2]);
    if (sk) {
      bcs1v_skew(code & 7, sk, ax, ay, az);
    } else {
      if (code & 4) ax = R(0);
      if (code & 2) ay = R(0);
      if (code & 1) az = R(0);
    }
  }
  const double dt05 = 0.5 * DT1;
  if (want_ek) {
    const double wx = (double)v.x + dt05 * (double)ax, wy = (double)v.y + dt05 * (double)ay,
                 wz = (double)v.z + dt05 * (double)az;
    ek = (wx * wx + wy * wy + wz * wz) * 0.5 * (double)ms;
  }
  // VELOCITY (velocity.F:56-62)
  const R dt12 = R(DT12);
  v.x = v.x + dt12 * ax; v.y = v.y + dt12 * ay; v.z = v.z + dt12 * az;
  // DEPLA (displacement.F:69-100), FP64 accumulation
  const double ux = DT2 * (double)v.x, uy = DT2 * (double)v.y, uz = DT2 * (double)v.z;
  qx = qx + ux; qy = qy + uy; qz = qz + uz;
  px = px + ux; py = py + uy; pz = pz + uz;
  if (rot) {
    const R in = w.w;
    if (in > R(0)) { const R r = R(1) / in; rx *= r; ry *= r; rz *= r; }
    else { rx = ry = rz = R(0); }
    if (sk) {
      bcs1v_skew((code >> 3) & 7, sk, w.x, w.y, w.z);
      bcs1v_skew((code >> 3) & 7, sk, rx, ry, rz);
    } else {
      if (code & 32) { w.x = R(0); rx = R(0); }
      if (code & 16) { w.y = R(0); ry = R(0); }
      if (code & 8)  { w.z = R(0); rz = R(0); }
    }
    if (code & 64) {
      const LinkMean* lm = &a.link_mean[a.link_of[n]];
      const int icr = lm->icr;
      if (icr & 4) rx = R(lm->ar[0]);
      if (icr & 2) ry = R(lm->ar[1]);
      if (icr & 1) rz = R(lm->ar[2]);
      if (sk) {
        bcs1v_skew((code >> 3) & 7, sk, rx, ry, rz);
      } else {
        if (code & 32) rx = R(0);
        if (code & 16) ry = R(0);
        if (code & 8)  rz = R(0);
      }
    }
    if (want_ek) {
      const double wx = (double)w.x + dt05 * (double)rx, wy = (double)w.y + dt05 * (double)ry,
                   wz = (double)w.z + dt05 * (double)rz;
      ekr = (wx * wx + wy * wy + wz * wz) * 0.5 * (double)in;
    }
    w.x = w.x + dt12 * rx; w.y = w.y + dt12 * ry; w.z = w.z + dt12 * rz;
  }
}

template <class R, int TILE>
__device__ __forceinline__ void node_pass(NodeArgs<R> a, int parity) {
  typedef typename Vec4<R>::T R4;
  __shared__ double s_e0[TILE / 32], s_e1[TILE / 32];
  const int* __restrict__ adsky = a.adsky;
  const R4* __restrict__ fslot = a.fslot;
  const R4* __restrict__ mslot = a.mslot;
  double4* __restrict__ X = a.X;
  R4* __restrict__ V = a.V;
  R4* __restrict__ VR = a.VR;
  double* __restrict__ DX = a.DX;
  double* __restrict__ DY = a.DY;
  double* __restrict__ DZ = a.DZ;
  const unsigned char* __restrict__ codes = a.code;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    // Node loads first, unconditionally: every part's node range is padded to whole
    // tiles, so n < nnodpad and padding nodes hold zeros (no slots, no mass).  They
    // are issued before the part descriptor arrives; `valid` gates the stores only.
    const int n = tile * TILE + threadIdx.x;
    const int k0 = adsky[n], k1 = adsky[n + 1];
    const double4 xm = X[n];
    R4 v = V[n];
    const unsigned char code = codes[n];
    const double dx = DX[n], dy = DY[n], dz = DZ[n];
    R4 f0 = mk4(R(0), R(0), R(0), R(0)), m0 = f0, w0 = f0;
    // VR is loaded before the rotational-node bit arrives (a dependent load would
    // lengthen the pass's latency chain); only rotational nodes use and write it
    const bool rn = rot_node(a, n);
    if (VR && (!a.rot_sparse || rn)) w0 = VR[n];
    const int part = a.tile_part[tile];
    const PartDesc pd = a.parts[part];
    const bool valid = n < pd.node_end;
    const PartTime t0 = a.time[parity * a.nparts + part];
    // the slots and the time-step reduction come from the element pass; a node's
    // first two slots are loaded together
    pdl_wait();
    pdl_trigger();
    R4 f1 = mk4(R(0), R(0), R(0), R(0)), m1 = f1;
    if (k1 > k0) f0 = fslot[k0];
    if (k1 > k0 + 1) f1 = fslot[k0 + 1];
    if (rn && mslot) {
      if (k1 > k0) m0 = mslot[k0];
      if (k1 > k0 + 1) m1 = mslot[k0 + 1];
    }
    PartAcc ac = a.acc[parity * a.nparts + part];
    if (a.halo_slot) {   // SPMD: time step = min over every rank's reduction (SPMD_GLOB_MIN5)
      for (int r = 0; r < a.nranks; ++r) {
        const PartAcc o = *reinterpret_cast<const PartAcc*>(a.xbuf + (size_t)r * a.xbytes + 2 * (size_t)a.nhalo * sizeof(R4));
        ac.dtkey = o.dtkey < ac.dtkey ? o.dtkey : ac.dtkey;
        ac.dtbits = o.dtbits < ac.dtbits ? o.dtbits : ac.dtbits;
      }
    }
    int ityp, nelt;
    double DT2;
    cycle_dt(ac, t0, a.growth, a.dtmx, a.split, DT2, ityp, nelt);
    const double DT1 = t0.dt2;
    const double DT12 = 0.5 * (DT1 + DT2);
    double ek = 0.0, ekr = 0.0;
    const bool rb = a.rb_role && a.rb_role[n];     // updated by rbody_kernel
    if (valid && !rb) {
      // ASSPAR4: the node's patch partials in ascending patch order
      R ax = f0.x, ay = f0.y, az = f0.z;
      if (k1 > k0 + 1) { ax += f1.x; ay += f1.y; az += f1.z; }
      for (int k = k0 + 2; k < k1; ++k) {
        const R4 f = fslot[k];
        ax += f.x; ay += f.y; az += f.z;
      }
      const int hs = a.halo_slot ? a.halo_slot[n] : -1;
      if (hs >= 0) {       // SPMD_EXCH_A: every rank's partial, in rank order
        for (int r = 0; r < a.nranks; ++r) {
          const R4 f = reinterpret_cast<const R4*>(a.xbuf + (size_t)r * a.xbytes)[hs];
          if (r == 0) { ax = f.x; ay = f.y; az = f.z; }
          else { ax += f.x; ay += f.y; az += f.z; }
        }
      }
      R rx = R(0), ry = R(0), rz = R(0);
      if (rn) {
        rx = m0.x; ry = m0.y; rz = m0.z;
        if (k1 > k0 + 1) { rx += m1.x; ry += m1.y; rz += m1.z; }
        for (int k = k0 + 2; k < k1; ++k) {
          const R4 m = mslot[k];
          rx += m.x; ry += m.y; rz += m.z;
        }
        if (hs >= 0) {
          for (int r = 0; r < a.nranks; ++r) {
            const R4 m = reinterpret_cast<const R4*>(a.xbuf + (size_t)r * a.xbytes)[a.nhalo + hs];
            if (r == 0) { rx = m.x; ry = m.y; rz = m.z; }
            else { rx += m.x; ry += m.y; rz += m.z; }
          }
        }
      }
      double px = xm.x, py = xm.y, pz = xm.z, qx = dx, qy = dy, qz = dz;
      R4 w = w0;
      node_update<R>(a, n, code, rn, ax, ay, az, rx, ry, rz, R(xm.w), DT1, DT2, DT12, px, py, pz,
                     qx, qy, qz, v, w, ek, ekr);
      V[n] = v;
      DX[n] = qx; DY[n] = qy; DZ[n] = qz;
      X[n] = make_double4(px, py, pz, xm.w);
      if (rn) VR[n] = w;
    }
    if (valid && a.halo_slot && !a.halo_ke[n]) { ek = 0.0; ekr = 0.0; }   // counted by another rank
    // per-tile kinetic energy partials (fixed tree order -> deterministic)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ek += __shfl_xor_sync(0xffffffffu, ek, o);
      ekr += __shfl_xor_sync(0xffffffffu, ekr, o);
    }
    if (lane == 0) { s_e0[warp] = ek; s_e1[warp] = ekr; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double s0 = 0.0, s1 = 0.0;
      for (int w = 0; w < TILE / 32; ++w) { s0 += s_e0[w]; s1 += s_e1[w]; }
      a.blk_ekin[tile] = s0;
      a.blk_ekinr[tile] = s1;
      if (tile == pd.tile_start) {
        PartTime t1;
        t1.tt = t0.tt + DT2; t1.dt2 = DT2; t1.dt2old = DT2; t1.dt1 = DT1; t1.dt12 = DT12;
        t1.ncycle = t0.ncycle + 1; t1.ityptst = ityp; t1.neltst = nelt; t1.pad = 0;
        a.time[(1 - parity) * a.nparts + part] = t1;
        PartAcc r; r.dtkey = ~0ull; r.dtbits = ~0ull;
        a.acc[(1 - parity) * a.nparts + part] = r;
      }
    }
    __syncthreads();
  }
}

// Two register budgets for the same pass: node_kernel leaves the budget to the
// compiler (a single wave is latency-bound and runs faster with more registers
// per thread); node_kernel_wide asks for 8 blocks of 128 per SM, for meshes of
// many node tiles, where the pass streams HBM and more loads in flight pay.
template <class R, int TILE>
__global__ void __launch_bounds__(TILE) node_kernel(NodeArgs<R> a, int parity) {
  node_pass<R, TILE>(a, parity);
}
// Resident threads per SM the wide form is compiled for (its register budget).  On
// the C4 mixed mesh (2.05 M nodes, split) 1024 (64 registers, 20 B spilled) ran
// the pass in 78.7 us per cycle, 1280 (48 registers, 96 B spilled) in 86.3 and 1536
// (40 registers, 128 B spilled) in 84.8 (eager cycles timed with events, B200).
#ifndef ORB_NODE_WIDE_THREADS
#define ORB_NODE_WIDE_THREADS 1024
#endif
template <class R, int TILE>
__global__ void __launch_bounds__(TILE, ORB_NODE_WIDE_THREADS / TILE) node_kernel_wide(NodeArgs<R> a, int parity) {
  node_pass<R, TILE>(a, parity);
}

// ===========================================================================
// loads (FORCE, force.F90, Parith/ON branch): one thread per load, at the time TT
// of the cycle's start and with the coordinates of the cycle's start; each load
// writes its own assembly slots.  External work per load (FP64, cumulative):
//  - /CLOAD: WFEXC = 1/2 (F(TT-DT1) + F(TT)) . v, times the cycle's DT2
//    (resol.F:6238).  DT2 is known only after the element pass, so the power is
//    kept in wpend and multiplied by DT2 at the next cycle's start;
//  - /PLOAD: DT1 F . (v1 + v2 + v3 [+ v4]).
// ===========================================================================
template <class R>
__global__ void __launch_bounds__(128)
load_kernel(const LoadDesc* __restrict__ loads, int nload, const FuncDesc* __restrict__ funcs,
            const double* __restrict__ fx, const double* __restrict__ fy, const R* __restrict__ skews,
            const PartTime* __restrict__ time, int parity, int nparts, const double4* __restrict__ X,
            const typename Vec4<R>::T* __restrict__ V, const typename Vec4<R>::T* __restrict__ VR,
            typename Vec4<R>::T* __restrict__ fslot, typename Vec4<R>::T* __restrict__ mslot,
            double* __restrict__ wacc, double* __restrict__ wpend) {
  typedef typename Vec4<R>::T R4;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nload) return;
  const LoadDesc L = loads[e];
  const PartTime t0 = time[parity * nparts + L.part];
  const FuncDesc F = funcs[L.func];
  const R ts = R(t0.tt), dt1 = R(t0.dt2);
  const R zero4 = R(0);
  if (L.type == 0) {
    const R a0 = R(L.fcy) * finter<R>(fx + F.first, fy + F.first, F.count, (ts - dt1) * R(L.fcx));
    const R aa = R(L.fcy) * finter<R>(fx + F.first, fy + F.first, F.count, ts * R(L.fcx));
    const bool rot = L.dir > 3;
    const int d = rot ? L.dir - 4 : L.dir - 1;
    const int n = L.node[0];
    const R4 vel = rot ? VR[n] : V[n];
    R f0 = zero4, f1 = zero4, f2 = zero4;
    R vv;
    if (L.skew < 0) {
      f0 = d == 0 ? aa : zero4; f1 = d == 1 ? aa : zero4; f2 = d == 2 ? aa : zero4;
      vv = d == 0 ? vel.x : d == 1 ? vel.y : vel.z;
    } else {
      const R* sk = skews + 9 * L.skew + 3 * d;
      vv = sk[0] * vel.x + sk[1] * vel.y + sk[2] * vel.z;
      f0 = sk[0] * aa; f1 = sk[1] * aa; f2 = sk[2] * aa;
    }
    const R4 fz = mk4(zero4, zero4, zero4, zero4), fv = mk4(f0, f1, f2, zero4);
    fslot[L.slot[0]] = rot ? fz : fv;
    if (mslot) mslot[L.slot[0]] = rot ? fv : fz;
    wacc[e] += wpend[e] * t0.dt2;
    wpend[e] = (double)(R(0.5) * (a0 + aa) * vv);
  } else {
    const R aa = R(L.fcy) * finter<R>(fx + F.first, fy + F.first, F.count, ts * R(L.fcx));
    const bool quad = L.dir == 4;
    // triangle: (x3 - x1) x (x3 - x2) / 6; its fourth node entry is a valid padding node
    const double4 x1 = X[L.node[0]], x2 = X[L.node[1]], x3 = X[L.node[2]], x4 = quad ? X[L.node[3]] : x3;
    const R ax = R(x3.x) - R(x1.x), ay = R(x3.y) - R(x1.y), az = R(x3.z) - R(x1.z);
    const R bx = R(x4.x) - R(x2.x), by = R(x4.y) - R(x2.y), bz = R(x4.z) - R(x2.z);
    const R NX = ay * bz - az * by, NY = az * bx - ax * bz, NZ = ax * by - ay * bx;
    const R c = quad ? R(0.125) : R(1.0 / 6.0);
    const R fxx = aa * NX * c, fyy = aa * NY * c, fzz = aa * NZ * c;
    const R4 fv = mk4(fxx, fyy, fzz, zero4), fz = mk4(zero4, zero4, zero4, zero4);
    R sv0 = zero4, sv1 = zero4, sv2 = zero4;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < L.dir) {
        fslot[L.slot[k]] = fv;
        if (mslot) mslot[L.slot[k]] = fz;
        const R4 v = V[L.node[k]];
        sv0 = sv0 + v.x; sv1 = sv1 + v.y; sv2 = sv2 + v.z;
      }
    }
    const R sv[3] = {sv0, sv1, sv2};
    wacc[e] += (double)(dt1 * (fxx * sv[0] + fyy * sv[1] + fzz * sv[2]));
  }
}

// ===========================================================================
// node input/output: one nodal array of a part between the caller's layout
// (3 doubles per node, node-major, staged in device memory) and the device
// layout.  kind: 0 X (keeps the mass in .w), 1 D, 2 V, 3 VR (keeps the inertia);
// to_device: 1 stage -> device arrays, 0 device arrays -> stage.
// ===========================================================================
template <class R>
__global__ void __launch_bounds__(256)
node_io_kernel(int kind, int to_device, double* __restrict__ stage, int n, int s, double4* X, double* DX,
               double* DY, double* DZ, typename Vec4<R>::T* V, typename Vec4<R>::T* VR) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* q = stage + 3 * (size_t)i;
  const int g = s + i;
  if (to_device) {
    const double a = q[0], b = q[1], c = q[2];
    if (kind == 0) X[g] = make_double4(a, b, c, X[g].w);
    else if (kind == 1) { DX[g] = a; DY[g] = b; DZ[g] = c; }
    else if (kind == 2) V[g] = mk4(R(a), R(b), R(c), R(0));
    else { const R w = VR[g].w; VR[g] = mk4(R(a), R(b), R(c), w); }
  } else {
    double a, b, c;
    if (kind == 0) { const double4 x = X[g]; a = x.x; b = x.y; c = x.z; }
    else if (kind == 1) { a = DX[g]; b = DY[g]; c = DZ[g]; }
    else if (kind == 2) { const typename Vec4<R>::T v = V[g]; a = v.x; b = v.y; c = v.z; }
    else { const typename Vec4<R>::T v = VR[g]; a = v.x; b = v.y; c = v.z; }
    q[0] = a; q[1] = b; q[2] = c;
  }
}

// ===========================================================================
// rigid links (RLINK1, rlink1.F): per link (one block), MASS = sum MS and
// AX = sum MS*A over its nodes after ACCELE and BCS10 (the node kernel's
// ASSPAR4 order), sums in FP64 in a fixed order; mean = AX / MASS.  Same for
// the rotations with IN.  Runs between the element kernels and the node kernel.
// ===========================================================================
constexpr int LINK_THREADS = 128;

template <class R>
__global__ void __launch_bounds__(LINK_THREADS)
link_kernel(const LinkDesc* __restrict__ links, const int* __restrict__ link_nodes, const int* __restrict__ adsky,
            const typename Vec4<R>::T* __restrict__ fslot, const typename Vec4<R>::T* __restrict__ mslot,
            const double4* __restrict__ X, const typename Vec4<R>::T* __restrict__ VR,
            const unsigned char* __restrict__ codes, const int* __restrict__ skew_of, const R* __restrict__ skews,
            LinkMean* __restrict__ out) {
  typedef typename Vec4<R>::T R4;
  __shared__ double s_sum[8][LINK_THREADS / 32];
  const LinkDesc L = links[blockIdx.x];
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (L.ic | L.icr) {
    for (int j = threadIdx.x; j < L.count; j += LINK_THREADS) {
      const int n = link_nodes[L.first + j];
      const int k0 = adsky[n], k1 = adsky[n + 1];
      const unsigned char code = codes[n];
      R ax = R(0), ay = R(0), az = R(0);
      if (k1 > k0) { const R4 f = fslot[k0]; ax = f.x; ay = f.y; az = f.z; }
      for (int k = k0 + 1; k < k1; ++k) { const R4 f = fslot[k]; ax += f.x; ay += f.y; az += f.z; }
      const R ms = R(X[n].w);
      if (ms > R(0)) { const R r = R(1) / ms; ax *= r; ay *= r; az *= r; }
      else { ax = ay = az = R(0); }
      const R* sk = (code & 128) ? skews + 9 * skew_of[n] : nullptr;
      if (sk) {
        bcs1v_skew(code & 7, sk, ax, ay, az);
      } else {
        if (code & 4) ax = R(0);
        if (code & 2) ay = R(0);
        if (code & 1) az = R(0);
      }
      s[0] += (double)ms; s[1] += (double)(ms * ax); s[2] += (double)(ms * ay); s[3] += (double)(ms * az);
      if (VR && mslot && L.icr) {
        R rx = R(0), ry = R(0), rz = R(0);
        if (k1 > k0) { const R4 m = mslot[k0]; rx = m.x; ry = m.y; rz = m.z; }
        for (int k = k0 + 1; k < k1; ++k) { const R4 m = mslot[k]; rx += m.x; ry += m.y; rz += m.z; }
        const R in = VR[n].w;
        if (in > R(0)) { const R r = R(1) / in; rx *= r; ry *= r; rz *= r; }
        else { rx = ry = rz = R(0); }
        if (sk) {
          bcs1v_skew((code >> 3) & 7, sk, rx, ry, rz);
        } else {
          if (code & 32) rx = R(0);
          if (code & 16) ry = R(0);
          if (code & 8)  rz = R(0);
        }
        s[4] += (double)in; s[5] += (double)(in * rx); s[6] += (double)(in * ry); s[7] += (double)(in * rz);
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], o);
    if (lane == 0) s_sum[q][warp] = s[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      t[q] = 0.0;
      for (int w = 0; w < LINK_THREADS / 32; ++w) t[q] += s_sum[q][w];
    }
    LinkMean r;
    r.ic = t[0] != 0.0 ? L.ic : 0;        // rlink1.F: IF(MASS==ZERO)GOTO 250
    r.icr = t[4] != 0.0 ? L.icr : 0;      // IF(INER==ZERO)RETURN
    for (int c = 0; c < 3; ++c) {
      r.a[c] = r.ic ? t[1 + c] / t[0] : 0.0;
      r.ar[c] = r.icr ? t[5 + c] / t[4] : 0.0;
    }
    out[blockIdx.x] = r;
  }
}

// ===========================================================================
// rigid bodies (/RBODY): RBYFOR -> RGBODFP (rgbodfp.F, explicit 3D, no rotational
// BCS on the main node), then, after ACCELE and BCS10 of the main node, RBYVIT ->
// RGBODV (rgbodv.F, more than two secondary nodes), VELOCITY and DEPLA of every
// node of the body, and its kinetic energy with the RBYCOR correction (rgbcor.F).
// One block per body, between the element pass and the node pass; the node pass
// leaves the bodies' nodes alone.
// ===========================================================================
struct RBodyDesc {
  int master;           // padded global node number of the main node
  int first, count;     // secondary nodes rb_nodes[first .. first+count-1]
  int part;
};
constexpr int RB_THREADS = 128;

template <class R>
__device__ inline void rotbmr_dev(const R* vr, R* rby, R dt) {
  const R rx = dt * vr[0], ry = dt * vr[1], rz = dt * vr[2];
  const R rx2 = rx * rx, ry2 = ry * ry, rz2 = rz * rz;
  const R r2 = fmax(R(1e-10), rx2 + ry2 + rz2);
  const R r = sqrt(r2);
  R c = cos(r);
  const R cm1 = R(1) - c;
  c = c * r2;
  const R s = sin(r) * r;
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
  R bn = sqrt(b11 * b11 + b21 * b21 + b31 * b31);
  b11 = b11 / bn; b21 = b21 / bn; b31 = b31 / bn;
  bn = sqrt(b12 * b12 + b22 * b22 + b32 * b32);
  b12 = b12 / bn; b22 = b22 / bn; b32 = b32 / bn;
  rby[0] = b11; rby[1] = b21; rby[2] = b31;
  rby[3] = b12; rby[4] = b22; rby[5] = b32;
  rby[6] = b21 * b32 - b31 * b22;
  rby[7] = b31 * b12 - b11 * b32;
  rby[8] = b11 * b22 - b21 * b12;
}

template <class R>
__global__ void __launch_bounds__(RB_THREADS)
rbody_kernel(NodeArgs<R> a, int parity, const RBodyDesc* __restrict__ bodies, const int* __restrict__ rb_nodes,
             R* rby_state, double* rb_ekin, double* rb_ekinr) {
  typedef typename Vec4<R>::T R4;
  __shared__ double s_sum[6][RB_THREADS / 32];
  __shared__ R s_am[3], s_vg[3], s_a[3];
  __shared__ double s_xm[3];
  __shared__ R s_vm[3];
  __shared__ double s_dt[3];     // DT1, DT2, DT12
  const RBodyDesc B = bodies[blockIdx.x];
  const int M = B.master;
  R* rby = rby_state + 12 * (size_t)blockIdx.x;
  const double4 xm4 = a.X[M];
  // ASSPAR4 sum of one node's slots, in ascending slot order
  auto raw = [&](int n, R* f, R* mo) {
    f[0] = f[1] = f[2] = mo[0] = mo[1] = mo[2] = R(0);
    const int k0 = a.adsky[n], k1 = a.adsky[n + 1];
    for (int k = k0; k < k1; ++k) {
      const R4 g = a.fslot[k];
      f[0] = f[0] + g.x; f[1] = f[1] + g.y; f[2] = f[2] + g.z;
      if (a.mslot) { const R4 h = a.mslot[k]; mo[0] = mo[0] + h.x; mo[1] = mo[1] + h.y; mo[2] = mo[2] + h.z; }
    }
  };
  // secondary nodes' forces and moments about the main node, FP64 partial sums
  double S[6] = {0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < B.count; i += RB_THREADS) {
    const int n = rb_nodes[B.first + i];
    R f[3], mo[3];
    raw(n, f, mo);
    const double4 xn = a.X[n];
    const R dx = R(xn.x - xm4.x), dy = R(xn.y - xm4.y), dz = R(xn.z - xm4.z);
    S[0] += (double)f[0]; S[1] += (double)f[1]; S[2] += (double)f[2];
    S[3] += (double)(mo[0] + dy * f[2] - dz * f[1]);
    S[4] += (double)(mo[1] + dz * f[0] - dx * f[2]);
    S[5] += (double)(mo[2] + dx * f[1] - dy * f[0]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) S[q] += __shfl_xor_sync(0xffffffffu, S[q], o);
    if (lane == 0) s_sum[q][warp] = S[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double T[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      T[q] = 0.0;
      for (int w = 0; w < RB_THREADS / 32; ++w) T[q] += s_sum[q][w];
    }
    const PartTime t0 = a.time[parity * a.nparts + B.part];
    const PartAcc ac = a.acc[parity * a.nparts + B.part];
    int ityp, nelt;
    double DT2;
    cycle_dt(ac, t0, a.growth, a.dtmx, a.split, DT2, ityp, nelt);
    const double DT1 = t0.dt2;
    const double DT12 = 0.5 * (DT1 + DT2);
    s_dt[0] = DT1; s_dt[1] = DT2; s_dt[2] = DT12;
    // the main node: its own slots plus the body's sums (phase 2), the frame and
    // the pseudo moment IN(M) * rotational acceleration
    R af[3], am[3];
    raw(M, af, am);
    for (int c = 0; c < 3; ++c) { af[c] = R((double)af[c] + T[c]); am[c] = R((double)am[c] + T[3 + c]); }
    const R4 wm = a.VR[M];              // .w = IN(M), the smallest principal inertia
    const R inm = wm.w;
    rby[9] = fmax(rby[9], inm); rby[10] = fmax(rby[10], inm); rby[11] = fmax(rby[11], inm);
    R vi[3];
    vi[0] = rby[0] * wm.x + rby[1] * wm.y + rby[2] * wm.z;
    vi[1] = rby[3] * wm.x + rby[4] * wm.y + rby[5] * wm.z;
    vi[2] = rby[6] * wm.x + rby[7] * wm.y + rby[8] * wm.z;
    rotbmr_dev(vi, rby, R(DT1));
    R p1 = rby[0] * am[0] + rby[1] * am[1] + rby[2] * am[2];
    R p2 = rby[3] * am[0] + rby[4] * am[1] + rby[5] * am[2];
    R p3 = rby[6] * am[0] + rby[7] * am[1] + rby[8] * am[2];
    p1 = p1 + (rby[10] - rby[11]) * vi[1] * vi[2];
    p2 = p2 + (rby[11] - rby[9]) * vi[2] * vi[0];
    p3 = p3 + (rby[9] - rby[10]) * vi[0] * vi[1];
    const R q1 = p1 * inm / rby[9], q2 = p2 * inm / rby[10], q3 = p3 * inm / rby[11];
    am[0] = rby[0] * q1 + rby[3] * q2 + rby[6] * q3;
    am[1] = rby[1] * q1 + rby[4] * q2 + rby[7] * q3;
    am[2] = rby[2] * q1 + rby[5] * q2 + rby[8] * q3;
    // ACCELE and BCS10 of the main node
    const R msm = R(xm4.w);
    R ax[3], ar[3];
    for (int c = 0; c < 3; ++c) {
      ax[c] = msm > R(0) ? af[c] * (R(1) / msm) : R(0);
      ar[c] = inm > R(0) ? am[c] * (R(1) / inm) : R(0);
    }
    if (!isfinite((double)ax[0] + (double)ax[1] + (double)ax[2])) raise_error(a.err, 6, M);
    R4 v = a.V[M], w = wm;
    const unsigned char code = a.code[M];
    const R* sk = (code & 128) ? a.skews + 9 * a.skew_of[M] : nullptr;
    if (sk) {
      bcs1v_skew(code & 7, sk, v.x, v.y, v.z);
      bcs1v_skew(code & 7, sk, ax[0], ax[1], ax[2]);
      bcs1v_skew((code >> 3) & 7, sk, w.x, w.y, w.z);
      bcs1v_skew((code >> 3) & 7, sk, ar[0], ar[1], ar[2]);
    } else {
      if (code & 4) { v.x = R(0); ax[0] = R(0); }
      if (code & 2) { v.y = R(0); ax[1] = R(0); }
      if (code & 1) { v.z = R(0); ax[2] = R(0); }
      if (code & 32) { w.x = R(0); ar[0] = R(0); }
      if (code & 16) { w.y = R(0); ar[1] = R(0); }
      if (code & 8)  { w.z = R(0); ar[2] = R(0); }
    }
    const R dt12 = R(DT12);
    s_vg[0] = w.x + ar[0] * dt12; s_vg[1] = w.y + ar[1] * dt12; s_vg[2] = w.z + ar[2] * dt12;
    s_a[0] = ax[0]; s_a[1] = ax[1]; s_a[2] = ax[2];
    s_vm[0] = v.x; s_vm[1] = v.y; s_vm[2] = v.z;
    s_xm[0] = xm4.x; s_xm[1] = xm4.y; s_xm[2] = xm4.z;
    // kinetic energy (ECRIT + RBYCOR): the body's mass on its main node, its
    // rotation in the principal frame
    const double dt05 = 0.5 * DT1;
    {
      const double vx = (double)v.x + dt05 * (double)ax[0], vy = (double)v.y + dt05 * (double)ax[1],
                   vz = (double)v.z + dt05 * (double)ax[2];
      rb_ekin[blockIdx.x] = (vx * vx + vy * vy + vz * vz) * 0.5 * (double)msm;
      const R h = R(dt05);
      const R w1 = w.x + ar[0] * h, w2 = w.y + ar[1] * h, w3 = w.z + ar[2] * h;
      const R i1 = rby[0] * w1 + rby[1] * w2 + rby[2] * w3;
      const R i2 = rby[3] * w1 + rby[4] * w2 + rby[5] * w3;
      const R i3 = rby[6] * w1 + rby[7] * w2 + rby[8] * w3;
      rb_ekinr[blockIdx.x] = 0.5 * ((double)rby[9] * (double)i1 * (double)i1 +
                                    (double)rby[10] * (double)i2 * (double)i2 +
                                    (double)rby[11] * (double)i3 * (double)i3);
    }
    s_am[0] = ar[0]; s_am[1] = ar[1]; s_am[2] = ar[2];
  }
  __syncthreads();
  const double DT2 = s_dt[1];
  const R dt12 = R(s_dt[2]), dt2 = R(DT2);
  const R usdt = R(1) / dt12;
  const R vg0 = s_vg[0], vg1 = s_vg[1], vg2 = s_vg[2];
  // RGBODV: the secondary nodes move with the body; then VELOCITY and DEPLA
  for (int i = threadIdx.x; i < B.count; i += RB_THREADS) {
    const int n = rb_nodes[B.first + i];
    R4 v = a.V[n], w = a.VR ? a.VR[n] : mk4(R(0), R(0), R(0), R(0));
    const unsigned char code = a.code[n];
    const R* sk = (code & 128) ? a.skews + 9 * a.skew_of[n] : nullptr;
    if (sk) {
      bcs1v_skew(code & 7, sk, v.x, v.y, v.z);
      bcs1v_skew((code >> 3) & 7, sk, w.x, w.y, w.z);
    } else {
      if (code & 4) v.x = R(0);
      if (code & 2) v.y = R(0);
      if (code & 1) v.z = R(0);
      if (code & 32) w.x = R(0);
      if (code & 16) w.y = R(0);
      if (code & 8)  w.z = R(0);
    }
    const R arx = (vg0 - w.x) * usdt, ary = (vg1 - w.y) * usdt, arz = (vg2 - w.z) * usdt;
    const double4 xn = a.X[n];
    const R dx = R(xn.x - s_xm[0]), dy = R(xn.y - s_xm[1]), dz = R(xn.z - s_xm[2]);
    const R v1x2 = vg0 * dy, v2x1 = vg1 * dx, v2x3 = vg1 * dz, v3x2 = vg2 * dy, v3x1 = vg2 * dx, v1x3 = vg0 * dz;
    const R vx1 = v2x3 - v3x2, vx2 = v3x1 - v1x3, vx3 = v1x2 - v2x1;
    const R ax = s_a[0] + (s_vm[0] + vx1 + R(0.5) * dt2 * (vg1 * vx3 - vg2 * vx2) - v.x) * usdt;
    const R ay = s_a[1] + (s_vm[1] + vx2 + R(0.5) * dt2 * (vg2 * vx1 - vg0 * vx3) - v.y) * usdt;
    const R az = s_a[2] + (s_vm[2] + vx3 + R(0.5) * dt2 * (vg0 * vx2 - vg1 * vx1) - v.z) * usdt;
    v.x = v.x + dt12 * ax; v.y = v.y + dt12 * ay; v.z = v.z + dt12 * az;
    a.V[n] = v;
    if (a.VR) {
      w.x = w.x + dt12 * arx; w.y = w.y + dt12 * ary; w.z = w.z + dt12 * arz;
      a.VR[n] = w;
    }
    const double ux = DT2 * (double)v.x, uy = DT2 * (double)v.y, uz = DT2 * (double)v.z;
    a.DX[n] = a.DX[n] + ux; a.DY[n] = a.DY[n] + uy; a.DZ[n] = a.DZ[n] + uz;
    a.X[n] = make_double4(xn.x + ux, xn.y + uy, xn.z + uz, xn.w);
  }
  __syncthreads();          // the secondary nodes read the main node's old state
  if (threadIdx.x == 0) {
    R4 v = a.V[M], w = a.VR[M];
    const unsigned char code = a.code[M];
    const R* sk = (code & 128) ? a.skews + 9 * a.skew_of[M] : nullptr;
    if (sk) {
      bcs1v_skew(code & 7, sk, v.x, v.y, v.z);
      bcs1v_skew((code >> 3) & 7, sk, w.x, w.y, w.z);
    } else {
      if (code & 4) v.x = R(0);
      if (code & 2) v.y = R(0);
      if (code & 1) v.z = R(0);
      if (code & 32) w.x = R(0);
      if (code & 16) w.y = R(0);
      if (code & 8)  w.z = R(0);
    }
    v.x = v.x + dt12 * s_a[0]; v.y = v.y + dt12 * s_a[1]; v.z = v.z + dt12 * s_a[2];
    w.x = w.x + dt12 * s_am[0]; w.y = w.y + dt12 * s_am[1]; w.z = w.z + dt12 * s_am[2];
    a.V[M] = v;
    a.VR[M] = w;
    const double ux = DT2 * (double)v.x, uy = DT2 * (double)v.y, uz = DT2 * (double)v.z;
    a.DX[M] = a.DX[M] + ux; a.DY[M] = a.DY[M] + uy; a.DZ[M] = a.DZ[M] + uz;
    a.X[M] = make_double4(s_xm[0] + ux, s_xm[1] + uy, s_xm[2] + uz, xm4.w);
  }
}

// ===========================================================================
// halo pack (domain decomposition): this rank's partial force and moment sums of
// every halo node it holds (its slots in ascending order, as the node kernel adds
// them), zero for halo nodes it does not hold, and its reduction of the cycle
// ===========================================================================
template <class R>
__global__ void __launch_bounds__(128)
halo_pack_kernel(const int* __restrict__ halo_node, const int* __restrict__ adsky,
                 const typename Vec4<R>::T* __restrict__ fslot, const typename Vec4<R>::T* __restrict__ mslot,
                 const PartAcc* __restrict__ acc, unsigned char* buf, int nhalo) {
  typedef typename Vec4<R>::T R4;
  R4* F = reinterpret_cast<R4*>(buf);
  R4* M = F + nhalo;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *reinterpret_cast<PartAcc*>(M + nhalo) = acc[0];
  if (i >= nhalo) return;
  const int n = halo_node[i];
  R4 f = mk4(R(0), R(0), R(0), R(0)), m = f;
  if (n >= 0) {
    const int k0 = adsky[n], k1 = adsky[n + 1];
    if (k1 > k0) {
      f = fslot[k0];
      if (mslot) m = mslot[k0];
    }
    for (int k = k0 + 1; k < k1; ++k) {
      const R4 a = fslot[k];
      f.x += a.x; f.y += a.y; f.z += a.z;
      if (mslot) { const R4 b = mslot[k]; m.x += b.x; m.y += b.y; m.z += b.z; }
    }
    f.w = R(0); m.w = R(0);
  }
  F[i] = f;
  M[i] = m;
}

}  // namespace orb
