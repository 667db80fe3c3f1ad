// ecycle.cu -- host implementation of the C-ABI declared in include/or_ecycle.h.
//
// finalize() turns the uploaded groups into the device layout:
//   * nodes of every part are concatenated, each part padded to NODE_TILE
//     nodes, X stored as double4 (x, y, z, nodal mass), V / VR as R4
//     (VR.w = rotational inertia), D as three FP64 planes, BCS codes as bytes;
//   * every element group is reordered along a Morton curve of the element
//     centroids and cut into patches of at most TILE elements; inside a patch
//     the elements are greedily coloured (no shared node within a colour) and
//     sorted by colour; connectivity becomes 16-bit patch-local node indices;
//   * each (patch, node) pair owns one slot of a node-major skyline; a node's
//     slots are ordered by patch number (element_pon_ ADSKY analogue).
// step() launches hex, shell and node kernels per cycle, replayed through a
// captured CUDA graph of GRAPH_CYCLES cycles.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <thread>
#include <utility>
#include <vector>
#include <array>

#include <nvtx3/nvToolsExt.h>

#include "../../include/or_ecycle.h"
#include "ecycle_kernels.cuh"
#include "persistent_kernel.cuh"
#include "adjoint_kernels.cuh"
#include "coqini_table.h"

using namespace orb;

namespace {

constexpr int NODE_TILE = 128;
constexpr int GRAPH_CYCLES = 32;


// ----------------------------------------------------------------------------
// host-side model as uploaded
// ----------------------------------------------------------------------------
struct HPart {
  int numnod = 0;
  std::vector<double> x, v, vr, ms, in;
  std::vector<int> icodt, icodr;
  std::vector<int> iskew;           // skew frame of the /BCS codes, -1 = global (may be empty)
  double ehour0 = 0, wpla0 = 0, wext0 = 0;   // cumulative energies before a restart
  int nel_solid = 0, nel_shell = 0;
  bool has_rot = false;
  int node_start = 0, node_pad = 0, tile_start = 0;
};
struct HLink {
  int part = 0, ic = 0, icr = 0;
  std::vector<int> nodes;           // part-local, 0-based
};
struct HRBody {                     // /RBODY after the starter's initialisation
  int part = 0, master = 0;         // part-local, 0-based
  std::vector<int> slaves;
  double rby[12];                   // principal axes e1, e2, e3, principal inertias
};
struct HLoad {                      // a /CLOAD node (type 0) or a /PLOAD segment (type 1)
  int type = 0, part = 0, func = 0, dir = 0, skew = -1;
  int node[4] = {-1, -1, -1, -1};   // part-local, 0-based
  double fcx = 1.0, fcy = 1.0;
};
struct HHex {
  int part = 0, nel = 0, gofs = 0;
  std::vector<int> conn;            // 8*nel, part-local
  or_material mat; or_solid_prop prop;
  std::vector<double> vol0;
  std::vector<int> internal;        // user element -> internal padded index
};
struct HShell {
  int part = 0, nel = 0, gofs = 0;
  std::vector<int> conn;            // 4*nel
  or_material mat; or_shell_prop prop;
  std::vector<double> thke, jca;
  std::vector<int> internal;
};

template <class T> struct DBuf {
  T* p = nullptr;
  size_t n = 0;
};

struct PatchSet {                   // host result of patch construction
  std::vector<PatchInfo> info;
  std::vector<int> nodes;           // global node ids, per patch contiguous
  std::vector<int> slots;           // slot id of each (patch, node)
  std::vector<int> elem_user;       // internal padded index -> (group, user index) encoded
  std::vector<int> elem_group;
  std::vector<uint16_t> local;      // internal padded index -> K local indices (+colour in corner 0)
  int nelpad = 0, nlmax = 0;
};

}  // namespace

struct or_ecycle {
  or_ecycle_config cfg{};
  std::string err;
  cudaStream_t stream = nullptr;
  std::vector<HPart> parts;
  std::vector<HHex> hex;
  std::vector<HShell> shell;
  std::vector<HLink> links;
  std::vector<HRBody> rbodies;
  std::vector<HLoad> loads;
  std::vector<std::vector<double>> fx, fy;   // time functions
  std::vector<std::array<double, 9>> skews;
  bool finalized = false;
  int tile_hex = 256, tile_shell = 256, tile_node = NODE_TILE;
  // device state
  void* impl = nullptr;
  void* adj = nullptr;               // adjoint workspace, allocated by the first or_ecycle_adjoint
  double phase_ms[4] = {0, 0, 0, 0};
  long long launches = 0;
  long long dev_bytes = 0;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t graph = nullptr;
  int last_code = 0, last_index = -1;
  int spmd_k = -1;                    // cycle index of a running domain-decomposed step, -1 outside one
  int next_parity = 0;                // time-buffer parity of the state after the last step
  bool pdl = true;                    // programmatic dependent launch of the cycle kernels
  int shell_staged = -1;              // staged 5-point shell kernel: -1 by wave count, 0 never, 1 always
  int nsm = 148;                      // multiprocessors of the device
  long long graph_launches = 0;       // kernel launches in one replay of graph_exec
};

namespace {

// NVTX range over a host call (tracing: nsys and ncu show the library's calls and
// phases on the timeline; NVTX is header-only and inert without a profiler)
struct Trace {
  explicit Trace(const char* name) { nvtxRangePushA(name); }
  ~Trace() { nvtxRangePop(); }
};

int fail(or_ecycle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

// The engine's IHBE (IPARG(23)) of a shell group from the starter's Ishell:
// 0 is the default 1 (hm_read_prop01.F:176), one integration point turns 2 into 1
// (:246-250), and GEO(171) maps 1, 2, 3, 4 to 1, 0, 2, 4 (:305-315, cgrtails.F:553).
int shell_ihbe(int ishell, int npt) {
  if (ishell == 0 || (npt == 1 && ishell == 2)) ishell = 1;
  return ishell == 1 ? 1 : ishell == 2 ? 0 : ishell == 3 ? 2 : 4;
}

#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(h, e_ == cudaErrorMemoryAllocation ? OR_E_NOMEM : OR_E_CUDA,    \
                  std::string(#call) + ": " + cudaGetErrorString(e_));            \
  } while (0)

template <class T>
int dalloc(or_ecycle* h, DBuf<T>& b, size_t n) {
  b.n = n;
  if (n == 0) { b.p = nullptr; return OR_OK; }
  CK(cudaMalloc((void**)&b.p, n * sizeof(T)));
  h->dev_bytes += (long long)(n * sizeof(T));
  return OR_OK;
}
template <class T>
int dput(or_ecycle* h, DBuf<T>& b, const std::vector<T>& v) {
  int rc = dalloc(h, b, v.size());
  if (rc) return rc;
  if (!v.empty()) CK(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return OR_OK;
}
template <class T> void dfree(DBuf<T>& b) { if (b.p) cudaFree(b.p); b.p = nullptr; b.n = 0; }

// check the kernels' compile-time 5-point rule against the shared table
constexpr bool coq5_matches_table() {
  for (int q = 0; q < 3; ++q)
    for (int ip = 0; ip < 5; ++ip)
      if (coq5(q, ip) != ZW_TABLE[4][11 * q + ip]) return false;
  return true;
}
static_assert(coq5_matches_table(), "5-point rule constants differ from COQINI's table");

uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  auto spread = [](uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
  };
  return spread(x) | (spread(y) << 1) | (spread(z) << 2);
}

// Builds patches for a list of groups of K-node elements.  conn_of(g) gives the
// part-local connectivity, node_base(g) the global node offset of the group's part.
template <int K, class GroupT>
int build_patches(or_ecycle* h, std::vector<GroupT>& groups, int tile, PatchSet& ps,
                  std::vector<std::vector<std::pair<int, int>>>& node_patch, int patch_base) {
  ps = PatchSet();
  int elem0 = 0;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    GroupT& g = groups[gi];
    const HPart& P = h->parts[g.part];
    const int nel = g.nel;
    // Morton order of centroids
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    std::vector<double> cen(3 * (size_t)nel);
    for (int e = 0; e < nel; ++e)
      for (int c = 0; c < 3; ++c) {
        double s = 0;
        for (int k = 0; k < K; ++k) s += P.x[3 * (size_t)g.conn[K * (size_t)e + k] + c];
        s /= K;
        cen[3 * (size_t)e + c] = s;
        lo[c] = std::min(lo[c], s); hi[c] = std::max(hi[c], s);
      }
    std::vector<uint64_t> code(nel);
    for (int e = 0; e < nel; ++e) {
      uint32_t q[3];
      for (int c = 0; c < 3; ++c) {
        double span = hi[c] - lo[c];
        double t = span > 0 ? (cen[3 * (size_t)e + c] - lo[c]) / span : 0.0;
        q[c] = (uint32_t)std::min(2097151.0, std::max(0.0, t * 2097151.0));
      }
      code[e] = morton3(q[0], q[1], q[2]);
    }
    std::vector<int> order(nel);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return code[a] < code[b]; });
    g.internal.assign(nel, -1);
    const int node_base = P.node_start;
    for (int s0 = 0; s0 < nel; s0 += tile) {
      const int n = std::min(tile, nel - s0);
      // unique nodes of the patch (sorted global ids)
      std::vector<int> nodes;
      nodes.reserve((size_t)n * K);
      for (int t = 0; t < n; ++t)
        for (int k = 0; k < K; ++k) nodes.push_back(node_base + g.conn[K * (size_t)order[s0 + t] + k]);
      std::sort(nodes.begin(), nodes.end());
      nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
      if ((int)nodes.size() > (int)LOCAL_MASK + 1)
        return fail(h, OR_E_UNSUPPORTED, "patch has more than 2048 distinct nodes");
      auto local_of = [&](int gid) { return (int)(std::lower_bound(nodes.begin(), nodes.end(), gid) - nodes.begin()); };
      // greedy colouring in Morton order
      std::vector<uint32_t> used(nodes.size(), 0u);
      std::vector<int> col(n);
      int ncol = 0;
      for (int t = 0; t < n; ++t) {
        uint32_t busy = 0;
        int lcs[K];
        for (int k = 0; k < K; ++k) { lcs[k] = local_of(node_base + g.conn[K * (size_t)order[s0 + t] + k]); busy |= used[lcs[k]]; }
        int c = 0;
        while (c < MAX_COLORS && (busy >> c & 1u)) ++c;
        if (c >= MAX_COLORS) return fail(h, OR_E_UNSUPPORTED, "more than 32 colours in a patch");
        col[t] = c;
        ncol = std::max(ncol, c + 1);
        for (int k = 0; k < K; ++k) used[lcs[k]] |= 1u << c;
      }
      std::vector<int> byc(n);
      std::iota(byc.begin(), byc.end(), 0);
      std::stable_sort(byc.begin(), byc.end(), [&](int a, int b) { return col[a] < col[b]; });
      PatchInfo pi{};
      pi.group = (int)gi; pi.nel = n; pi.node_ofs = (int)ps.nodes.size(); pi.nloc = (int)nodes.size();
      pi.ncolor = ncol; pi.elem0 = elem0; pi.part = g.part;
      const int pid = (int)ps.info.size();
      ps.info.push_back(pi);
      ps.nlmax = std::max(ps.nlmax, (int)nodes.size());
      for (size_t j = 0; j < nodes.size(); ++j) {
        node_patch[nodes[j]].push_back({patch_base + pid, (int)(ps.nodes.size() + j)});
      }
      ps.nodes.insert(ps.nodes.end(), nodes.begin(), nodes.end());
      ps.local.resize((size_t)(elem0 + tile) * K, 0);
      ps.elem_user.resize(elem0 + tile, -1);
      ps.elem_group.resize(elem0 + tile, -1);
      for (int t = 0; t < n; ++t) {
        const int ue = order[s0 + byc[t]];
        const int ie = elem0 + t;
        g.internal[ue] = ie;
        ps.elem_user[ie] = ue;
        ps.elem_group[ie] = (int)gi;
        for (int k = 0; k < K; ++k) {
          int l = local_of(node_base + g.conn[K * (size_t)ue + k]);
          if (k == 0) l |= col[byc[t]] << COLOR_SHIFT;
          ps.local[(size_t)ie * K + k] = (uint16_t)l;
        }
      }
      elem0 += tile;
    }
  }
  ps.nelpad = elem0;
  ps.slots.assign(ps.nodes.size(), -1);
  return OR_OK;
}

// Incidence lists of every patch at a fixed stride: nlmax+1 offsets, then for each
// patch node the corners (t: element of the patch, k: corner) that touch it, in
// ascending (t, k) order, each stored as its offset k*tile + t in a corner-force
// plane of the patch kernels.  The kernels sum a node's corner forces in this order.
int incidence_stride(const PatchSet& ps, int K, int tile) {
  const int s = ps.nlmax + 1 + K * tile;
  return (s + 7) & ~7;   // 16-byte rows: the hexa kernel stages them by bulk copy
}
void incidence_lists(const PatchSet& ps, int K, int tile, std::vector<uint16_t>& inc) {
  const size_t np = ps.info.size(), S = (size_t)incidence_stride(ps, K, tile), L = (size_t)ps.nlmax;
  inc.assign(np * S, 0);
  for (size_t p = 0; p < np; ++p) {
    const PatchInfo& pi = ps.info[p];
    uint16_t* ofs = &inc[p * S];
    uint16_t* ent = ofs + L + 1;
    std::vector<int> cnt(L + 1, 0);
    for (int t = 0; t < pi.nel; ++t)
      for (int k = 0; k < K; ++k) cnt[(ps.local[(size_t)(pi.elem0 + t) * K + k] & LOCAL_MASK) + 1]++;
    for (size_t j = 0; j < L; ++j) cnt[j + 1] += cnt[j];
    for (size_t j = 0; j <= L; ++j) ofs[j] = (uint16_t)cnt[j];
    for (int t = 0; t < pi.nel; ++t)
      for (int k = 0; k < K; ++k) {
        const int l = ps.local[(size_t)(pi.elem0 + t) * K + k] & LOCAL_MASK;
        ent[cnt[l]++] = (uint16_t)(k * tile + t);
      }
  }
}

// Patch node and slot lists at a fixed stride of nlmax entries per patch; the
// padding repeats the patch's first node (a valid address) with slot -1.
void padded_lists(const PatchSet& ps, std::vector<int>& nodes, std::vector<int>& slots) {
  const size_t np = ps.info.size(), L = (size_t)ps.nlmax;
  nodes.assign(np * L, 0);
  slots.assign(np * L, -1);
  for (size_t p = 0; p < np; ++p) {
    const PatchInfo& pi = ps.info[p];
    for (int j = 0; j < (int)L; ++j) {
      const int src = pi.node_ofs + (j < pi.nloc ? j : 0);
      nodes[p * L + j] = ps.nodes[src];
      if (j < pi.nloc) slots[p * L + j] = ps.slots[src];
    }
  }
}

// ----------------------------------------------------------------------------
// device model, templated on the element precision
// ----------------------------------------------------------------------------
template <class R>
struct Impl {
  typedef typename Vec4<R>::T R4;
  int nnodpad = 0, ntiles = 0, nparts = 0, nslot = 0;
  bool any_rot = false;
  bool any_corot = false;    // a hexa group in the convected frame (JCVT /= 0)
  // nodes
  DBuf<double4> X; DBuf<double> DX, DY, DZ; DBuf<R4> V, VR; DBuf<unsigned char> code;
  DBuf<unsigned> rotmask; std::vector<unsigned> rotmask_h;   // NodeArgs::rotmask, and its host copy
  int rot_sparse = 0;                                         // NodeArgs::rot_sparse
  DBuf<int> adsky, tile_part; DBuf<PartDesc> partd;
  DBuf<R4> fslot, mslot;
  DBuf<PartTime> time; DBuf<PartAcc> acc; DBuf<ErrorWord> err;
  DBuf<double> ekin, ekinr;
  // hexas
  PatchSet hps;
  DBuf<PatchInfo> hpatch; DBuf<HexGroupDesc> hdesc; DBuf<int> hnodes, hslots, helem; DBuf<uint4> hconn;
  DBuf<uint16_t> hinc, sinc;
  int hinc_stride = 0, sinc_stride = 0;
  DBuf<R> hsig, heint, hrho, hqvis, hpla, hepsd, hvol0; DBuf<double> hvol0dp;
  DBuf<double> hehour, hwpla;
  // shells
  PatchSet sps;
  DBuf<PatchInfo> spatch; DBuf<ShellGroupDesc> sdesc; DBuf<int> snodes, sslots, selem, sdegen; DBuf<uint2> sconn;
  DBuf<R> ssig, spla, sthk, sthke, shourg, seint, sjca;
  DBuf<double> sehour, swpla;
  DBuf<float> zw;
  int maxnpt = 1;
  int uniform_npt = 0;       // 5 when every shell group has 5 points, IHBE 1 and IPLA 0 (the kernels
                             // specialised for that form), else 0 (the general kernels)
  // domain decomposition: halo nodes of this rank's part
  DBuf<int> halo_slot, halo_node; DBuf<unsigned char> halo_ke;
  int nhalo = -1;            // -1: no halo set
  // rigid links
  DBuf<LinkDesc> linkd; DBuf<int> link_nodes, link_of; DBuf<LinkMean> link_mean;
  int nlinks = 0;
  // rigid bodies: descriptors, secondary nodes, frames (12 R per body), node roles,
  // per-body kinetic energies of the last cycle
  DBuf<RBodyDesc> rbd; DBuf<int> rb_nodes; DBuf<R> rby; DBuf<unsigned char> rb_role; DBuf<double> rb_ek, rb_ekr;
  std::vector<R> rby0;
  int nrb = 0;
  // staging of one nodal array of one part (3 doubles per node) for set/get_nodes
  DBuf<double> stage;
  // loads, time functions, skew frames
  DBuf<LoadDesc> loadd; DBuf<FuncDesc> funcd; DBuf<double> funcx, funcy, wacc, wpend;
  DBuf<R> skw; DBuf<int> skew_of;
  int nload = 0;
  // persistent launch (one part of shells whose state fits on the chip)
  struct Persist {
    bool on = false;
    int G = 0, P = 0, ncmax = 0;
    int T = 0;                 // threads per CTA
    int stall_cta = -1;        // test hook, OR_ECYCLE_TEST_STALL_CTA
    size_t smem = 0;
    DBuf<int> node_ofs, node_glob; DBuf<unsigned char> owner; DBuf<uint2> pconn;
    DBuf<R4> fslot2, mslot2; DBuf<PartAcc> acc3; DBuf<double> ek, ekr; DBuf<unsigned> sync;
  } per;

  HexArgs<R> hargs() {
    HexArgs<R> a;
    a.patch = hpatch.p; a.groups = hdesc.p; a.patch_nodes = hnodes.p; a.patch_slots = hslots.p;
    a.conn = hconn.p; a.elem_id = helem.p; a.X = X.p; a.V = V.p;
    a.sig = hsig.p; a.eint = heint.p; a.rho = hrho.p; a.qvis = hqvis.p; a.pla = hpla.p; a.epsd = hepsd.p;
    a.vol0 = hvol0.p; a.vol0dp = hvol0dp.p; a.fslot = fslot.p; a.time = time.p; a.acc = acc.p;
    a.blk_ehour = hehour.p; a.blk_wpla = hwpla.p; a.err = err.p;
    a.nelpad = hps.nelpad; a.nparts = nparts; a.npatch = (int)hps.info.size(); a.nlmax = hps.nlmax;
    a.inc = hinc.p; a.inc_stride = hinc_stride;
    return a;
  }
  ShellArgs<R> sargs() {
    ShellArgs<R> a;
    a.patch = spatch.p; a.groups = sdesc.p; a.patch_nodes = snodes.p; a.patch_slots = sslots.p;
    a.conn = sconn.p; a.elem_id = selem.p; a.degen = sdegen.p; a.X = X.p; a.V = V.p; a.VR = VR.p;
    a.sig = ssig.p; a.pla = spla.p; a.thk = sthk.p; a.thke = sthke.p; a.hourg = shourg.p; a.eint = seint.p;
    a.jca = sjca.p; a.fslot = fslot.p; a.mslot = mslot.p; a.time = time.p; a.acc = acc.p;
    a.blk_ehour = sehour.p; a.blk_wpla = swpla.p; a.err = err.p;
    a.nelpad = sps.nelpad; a.nparts = nparts; a.npatch = (int)sps.info.size(); a.maxnpt = maxnpt;
    a.nlmax = sps.nlmax;
    a.inc = sinc.p; a.inc_stride = sinc_stride;
    return a;
  }
  NodeArgs<R> nargs(const or_ecycle* h) {
    NodeArgs<R> a;
    a.parts = partd.p; a.tile_part = tile_part.p; a.adsky = adsky.p; a.fslot = fslot.p; a.mslot = mslot.p;
    a.X = X.p; a.DX = DX.p; a.DY = DY.p; a.DZ = DZ.p; a.V = V.p; a.VR = VR.p; a.code = code.p;
    a.time = time.p; a.acc = acc.p; a.blk_ekin = ekin.p; a.blk_ekinr = ekinr.p; a.err = err.p;
    a.growth = h->cfg.dt_growth; a.dtmx = h->cfg.dtmx; a.ntiles = ntiles; a.nparts = nparts;
    a.split = sizeof(R) == 4;
    a.halo_slot = nullptr; a.halo_ke = nullptr; a.xbuf = nullptr; a.xbytes = 0; a.nranks = 0; a.nhalo = 0;
    a.link_of = nlinks ? link_of.p : nullptr; a.link_mean = nlinks ? link_mean.p : nullptr;
    a.skew_of = skew_of.p; a.skews = skw.p;
    a.rb_role = nrb ? rb_role.p : nullptr;
    a.rotmask = any_rot ? rotmask.p : nullptr;
    a.rot_sparse = rot_sparse;
    return a;
  }
  void free_all() {
    dfree(X); dfree(DX); dfree(DY); dfree(DZ); dfree(V); dfree(VR); dfree(code); dfree(adsky); dfree(tile_part);
    dfree(rotmask);
    dfree(partd); dfree(fslot); dfree(mslot); dfree(time); dfree(acc); dfree(err); dfree(ekin); dfree(ekinr);
    dfree(hinc); dfree(sinc);
    dfree(hpatch); dfree(hdesc); dfree(hnodes); dfree(hslots); dfree(helem); dfree(hconn); dfree(hsig); dfree(heint);
    dfree(hrho); dfree(hqvis); dfree(hpla); dfree(hepsd); dfree(hvol0); dfree(hvol0dp); dfree(hehour); dfree(hwpla);
    dfree(spatch); dfree(sdesc); dfree(snodes); dfree(sslots); dfree(selem); dfree(sdegen); dfree(sconn);
    dfree(ssig); dfree(spla); dfree(sthk); dfree(sthke); dfree(shourg); dfree(seint); dfree(sjca);
    dfree(sehour); dfree(swpla); dfree(zw);
    dfree(halo_slot); dfree(halo_node); dfree(halo_ke);
    dfree(linkd); dfree(link_nodes); dfree(link_of); dfree(link_mean); dfree(stage);
    dfree(rbd); dfree(rb_nodes); dfree(rby); dfree(rb_role); dfree(rb_ek); dfree(rb_ekr);
    dfree(loadd); dfree(funcd); dfree(funcx); dfree(funcy); dfree(wacc); dfree(wpend); dfree(skw); dfree(skew_of);
    dfree(per.node_ofs); dfree(per.node_glob); dfree(per.owner); dfree(per.pconn); dfree(per.fslot2);
    dfree(per.mslot2); dfree(per.acc3); dfree(per.ek); dfree(per.ekr); dfree(per.sync);
  }
  PersistArgs pargs() {
    PersistArgs a;
    a.node_ofs = per.node_ofs.p; a.node_glob = per.node_glob.p; a.owner = per.owner.p; a.pconn = per.pconn.p;
    a.fslot2 = per.fslot2.p; a.mslot2 = per.mslot2.p; a.acc3 = per.acc3.p; a.ek_node = per.ek.p;
    a.ekr_node = per.ekr.p; a.sync = per.sync.p; a.patches_per_cta = per.P; a.ncmax = per.ncmax;
    a.ntiles_node = ntiles;
    a.stall_cta = per.stall_cta;
    return a;
  }
};

// dynamic shared memory of a patch kernel.  Hexa: the layout of hex_smem_bytes.
// Shell: for the NPT-point kernels the staged integration-point planes (6 NPT of
// TILE), then node planes (x, y, z in FP64; velocities and rotational velocities in
// R), 24 planes of TILE corner forces, the incidence lists.
template <class R>
size_t hex_smem(int nl, int tile, int inc_stride) {
  return hex_smem_bytes<R>(nl, tile, inc_stride);
}
template <class R>
size_t shell_smem(int nl, int tile, int inc_stride, int npt = 0) {
  return (size_t)shell_staged_planes(npt) * tile * sizeof(R) + (size_t)nl * (3 * sizeof(double) + 6 * sizeof(R)) +
         24 * (size_t)tile * sizeof(R) + 2 * (size_t)inc_stride;
}

// A cycle kernel launch; with pdl, programmatic stream serialization lets its
// blocks start before the previous kernel in the stream has finished (the
// kernels' pdl_wait / pdl_trigger protocol keeps every read ordered).  Only the
// element and node passes of the regular cycle use it: their alternation is what
// the protocol relies on.
template <class... P, class... A>
cudaError_t launch_k(void (*k)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t s, bool pdl,
                     A&&... args) {
  cudaLaunchConfig_t c{};
  c.gridDim = dim3(grid);
  c.blockDim = dim3(block);
  c.dynamicSmemBytes = smem;
  c.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  c.attrs = at;
  c.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&c, k, std::forward<A>(args)...);
}

template <class R, int T>
int launch_hex(or_ecycle* h, Impl<R>& m, int parity, bool pdl = false) {
  if (m.hps.info.empty()) return OR_OK;
  size_t sm = hex_smem<R>(m.hps.nlmax, T, m.hinc_stride);
  const unsigned g = (unsigned)m.hps.info.size();
  if (m.any_corot) CK(launch_k(hex_patch_kernel<R, T, 1>, g, T, sm, h->stream, pdl, m.hargs(), parity));
  else CK(launch_k(hex_patch_kernel<R, T, 0>, g, T, sm, h->stream, pdl, m.hargs(), parity));
  h->launches++;
  return OR_OK;
}
template <class R, int T, int NPT, bool STG>
int launch_shell(or_ecycle* h, Impl<R>& m, int parity, bool pdl) {
  if (m.sps.info.empty()) return OR_OK;
  size_t sm = shell_smem<R>(m.sps.nlmax, T, m.sinc_stride, STG ? NPT : 0);
  CK(launch_k(shell_patch_kernel<R, T, NPT, STG>, (unsigned)m.sps.info.size(), T, sm, h->stream, pdl, m.sargs(),
              parity, (const float*)m.zw.p));
  h->launches++;
  return OR_OK;
}
// The 5-point form with staged integration-point state where the shell patches
// exceed one wave of the register-held form (split precision)
// (OR_ECYCLE_SHELL_STAGED=0 never, =1 always, read at create)
template <class R>
bool shell_staged(const or_ecycle* h, const Impl<R>& m) {
  if (sizeof(R) != 4 || m.uniform_npt != 5 || h->shell_staged == 0) return false;
  return h->shell_staged == 1 ||
         (long long)m.sps.info.size() > (long long)h->nsm * min_blocks(Occupancy<R>::shell, h->tile_shell);
}
template <class R, int T>
int launch_shell_npt(or_ecycle* h, Impl<R>& m, int parity, bool pdl = false) {
  if (m.uniform_npt != 5) return launch_shell<R, T, 0, false>(h, m, parity, pdl);
  if constexpr (sizeof(R) == 4) {
    if (shell_staged(h, m)) return launch_shell<R, T, 5, true>(h, m, parity, pdl);
  }
  return launch_shell<R, T, 5, false>(h, m, parity, pdl);
}
template <class R>
int launch_link(or_ecycle* h, Impl<R>& m) {
  if (!m.nlinks) return OR_OK;
  link_kernel<R><<<(unsigned)m.nlinks, LINK_THREADS, 0, h->stream>>>(
      m.linkd.p, m.link_nodes.p, m.adsky.p, m.fslot.p, m.mslot.p, m.X.p, m.VR.p, m.code.p, m.skew_of.p, m.skw.p,
      m.link_mean.p);
  CK(cudaGetLastError());
  h->launches++;
  return OR_OK;
}
template <class R>
int launch_rbody(or_ecycle* h, Impl<R>& m, int parity) {
  if (!m.nrb) return OR_OK;
  rbody_kernel<R><<<(unsigned)m.nrb, RB_THREADS, 0, h->stream>>>(m.nargs(h), parity, m.rbd.p, m.rb_nodes.p, m.rby.p,
                                                                  m.rb_ek.p, m.rb_ekr.p);
  CK(cudaGetLastError());
  h->launches++;
  return OR_OK;
}
template <class R>
int launch_loads(or_ecycle* h, Impl<R>& m, int parity) {
  if (!m.nload) return OR_OK;
  load_kernel<R><<<(unsigned)((m.nload + 127) / 128), 128, 0, h->stream>>>(
      m.loadd.p, m.nload, m.funcd.p, m.funcx.p, m.funcy.p, m.skw.p, m.time.p, parity, m.nparts, m.X.p, m.V.p, m.VR.p,
      m.fslot.p, m.mslot.p, m.wacc.p, m.wpend.p);
  CK(cudaGetLastError());
  h->launches++;
  return OR_OK;
}
// node tiles beyond one wave of node_kernel_wide (1024 threads per SM): the
// streaming form
template <class R>
bool node_wide(const or_ecycle* h, const Impl<R>& m) {
  return m.ntiles > (long long)h->nsm * (1024 / NODE_TILE);
}
template <class R>
int launch_node(or_ecycle* h, Impl<R>& m, int parity, bool pdl = false) {
  const unsigned g = (unsigned)m.ntiles;
  if (node_wide(h, m))
    CK(launch_k(node_kernel_wide<R, NODE_TILE>, g, NODE_TILE, 0, h->stream, pdl, m.nargs(h), parity));
  else
    CK(launch_k(node_kernel<R, NODE_TILE>, g, NODE_TILE, 0, h->stream, pdl, m.nargs(h), parity));
  h->launches++;
  return OR_OK;
}

template <class F>
cudaError_t set_smem(F* f, int bytes) {
  return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <class R>
int set_smem_attrs(or_ecycle* h, Impl<R>& m) {
  int hs = (int)hex_smem<R>(m.hps.nlmax, h->tile_hex, m.hinc_stride);
  int ss = (int)shell_smem<R>(m.sps.nlmax, h->tile_shell, m.sinc_stride, 5);   // the largest: the 5-point kernels
  if (hs > 200 * 1024 || ss > 200 * 1024) return fail(h, OR_E_UNSUPPORTED, "patch shared memory above 200 KB");
  CK(set_smem(hex_patch_kernel<R, 64, 0>, hs));
  CK(set_smem(hex_patch_kernel<R, 128, 0>, hs));
  CK(set_smem(hex_patch_kernel<R, 256, 0>, hs));
  CK(set_smem(hex_patch_kernel<R, 64, 1>, hs));
  CK(set_smem(hex_patch_kernel<R, 128, 1>, hs));
  CK(set_smem(hex_patch_kernel<R, 256, 1>, hs));
  CK(set_smem(shell_patch_kernel<R, 64, 0, false>, ss));
  CK(set_smem(shell_patch_kernel<R, 128, 0, false>, ss));
  CK(set_smem(shell_patch_kernel<R, 256, 0, false>, ss));
  CK(set_smem(shell_patch_kernel<R, 64, 5, false>, ss));
  CK(set_smem(shell_patch_kernel<R, 128, 5, false>, ss));
  CK(set_smem(shell_patch_kernel<R, 256, 5, false>, ss));
  if constexpr (sizeof(R) == 4) {
    CK(set_smem(shell_patch_kernel<R, 64, 5, true>, ss));
    CK(set_smem(shell_patch_kernel<R, 128, 5, true>, ss));
    CK(set_smem(shell_patch_kernel<R, 256, 5, true>, ss));
  }
  return OR_OK;
}

// ----------------------------------------------------------------------------
// persistent launch: eligibility, layout, launch
// ----------------------------------------------------------------------------
template <class R>
using PersistFn = void (*)(ShellArgs<R>, NodeArgs<R>, PersistArgs, int, int, const float*);

template <class R>
PersistFn<R> persist_fn(int tile, bool npt5) {
  if (tile == 64) return npt5 ? shell_persistent_kernel<R, 64, 5> : shell_persistent_kernel<R, 64, 0>;
  if (tile == 128) return npt5 ? shell_persistent_kernel<R, 128, 5> : shell_persistent_kernel<R, 128, 0>;
  return npt5 ? shell_persistent_kernel<R, 256, 5> : shell_persistent_kernel<R, 256, 0>;
}

// Sets up the persistent launch when the handle qualifies: step() through a graph
// (cfg.graph != 0), one part, shell groups only, no rigid links and no /CLOAD or
// /PLOAD loads (the group pressure is fine), cfg.persistent not negative and
// OR_ECYCLE_PERSISTENT not 0, and the
// patches fit one cooperative wave of at most PERSIST_THREADS threads per CTA.
// Each CTA takes P consecutive patches (Morton order keeps them compact) and holds
// every node they touch; nodes no element touches are spread over the CTAs.
template <class R>
int persist_build(or_ecycle* h, Impl<R>& m) {
  auto& q = m.per;
  q.on = false;
  if (h->cfg.persistent < 0) return OR_OK;
  if (const char* s = std::getenv("OR_ECYCLE_PERSISTENT"))
    if (std::atoi(s) == 0) return OR_OK;
  if (!h->cfg.graph || m.nparts != 1 || !h->hex.empty() || h->shell.empty() || !h->links.empty() || m.nload ||
      !h->rbodies.empty())
    return OR_OK;
  const PatchSet& ps = m.sps;
  const int tile = h->tile_shell;
  const int npatch = (int)ps.info.size();
  const int P = std::max((npatch + h->nsm - 1) / h->nsm, (128 + tile - 1) / tile);
  if (P * tile > PERSIST_THREADS) return OR_OK;
  const int G = (npatch + P - 1) / P;
  std::vector<std::vector<int>> lists(G);
  std::vector<char> held(m.nnodpad, 0);
  for (int c = 0; c < G; ++c) {
    for (int p = c * P; p < std::min(npatch, (c + 1) * P); ++p)
      for (int j = 0; j < ps.info[p].nloc; ++j) lists[c].push_back(ps.nodes[ps.info[p].node_ofs + j]);
    std::sort(lists[c].begin(), lists[c].end());
    lists[c].erase(std::unique(lists[c].begin(), lists[c].end()), lists[c].end());
    for (int g : lists[c]) held[g] = 1;
  }
  const HPart& Pt = h->parts[0];
  for (int i = 0, k = 0; i < Pt.numnod; ++i)
    if (!held[Pt.node_start + i]) lists[(k++) % G].push_back(Pt.node_start + i);
  std::vector<int> ofs(G + 1, 0), glob;
  std::vector<unsigned char> own;
  std::vector<int> first(m.nnodpad, -1);
  int ncmax = 0;
  for (int c = 0; c < G; ++c) {
    std::sort(lists[c].begin(), lists[c].end());
    ncmax = std::max(ncmax, (int)lists[c].size());
    for (int g : lists[c]) {
      glob.push_back(g);
      own.push_back(first[g] < 0 ? 1 : 0);
      if (first[g] < 0) first[g] = c;
    }
    ofs[c + 1] = (int)glob.size();
  }
  if (ncmax > 65535) return OR_OK;
  std::vector<uint2> pconn((size_t)ps.nelpad, make_uint2(0, 0));
  for (int c = 0; c < G; ++c) {
    const std::vector<int>& L = lists[c];
    for (int p = c * P; p < std::min(npatch, (c + 1) * P); ++p) {
      const PatchInfo& pi = ps.info[p];
      for (int t = 0; t < pi.nel; ++t) {
        unsigned l[4];
        for (int k = 0; k < 4; ++k) {
          const int g = ps.nodes[pi.node_ofs + (ps.local[(size_t)(pi.elem0 + t) * 4 + k] & LOCAL_MASK)];
          l[k] = (unsigned)(std::lower_bound(L.begin(), L.end(), g) - L.begin());
        }
        pconn[(size_t)pi.elem0 + t] = make_uint2(l[0] | l[1] << 16, l[2] | l[3] << 16);
      }
    }
  }
  const size_t smem = persist_smem<R>(ncmax, tile, P, m.sinc_stride, ps.nlmax);
  if (smem > 200 * 1024) return OR_OK;
  // one thread per element, and per held node where the CTA holds more nodes than
  // elements (a node phase of one node per thread), in whole TILE groups
  const int T = std::min(PERSIST_THREADS / tile * tile, std::max(P * tile, (ncmax + tile - 1) / tile * tile));
  const PersistFn<R> fn = persist_fn<R>(tile, m.uniform_npt == 5);
  CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int nb = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, T, smem));
  if (nb < 1 || G > nb * h->nsm) return OR_OK;
  int rc;
  if ((rc = dput(h, q.node_ofs, ofs)) || (rc = dput(h, q.node_glob, glob)) || (rc = dput(h, q.owner, own)) ||
      (rc = dput(h, q.pconn, pconn)) || (rc = dalloc(h, q.fslot2, (size_t)m.nslot)) ||
      (rc = dalloc(h, q.mslot2, (size_t)m.nslot)) || (rc = dalloc(h, q.acc3, 3)) || (rc = dalloc(h, q.sync, 2)) ||
      (rc = dput(h, q.ek, std::vector<double>(m.nnodpad, 0.0))) ||
      (rc = dput(h, q.ekr, std::vector<double>(m.nnodpad, 0.0))))
    return rc;
  q.stall_cta = -1;
  if (const char* st = std::getenv("OR_ECYCLE_TEST_STALL_CTA")) q.stall_cta = std::atoi(st);
  q.on = true;
  q.G = G; q.P = P; q.T = T; q.ncmax = ncmax; q.smem = smem;
  return OR_OK;
}

// ncycles cycles in one cooperative launch, from the time state of parity0
template <class R>
int launch_persistent(or_ecycle* h, Impl<R>& m, int ncycles, int parity0) {
  auto& q = m.per;
  CK(cudaMemsetAsync(q.sync.p, 0, 2 * sizeof(unsigned), h->stream));
  CK(cudaMemsetAsync(q.acc3.p, 0xff, 3 * sizeof(PartAcc), h->stream));
  ShellArgs<R> sa = m.sargs();
  NodeArgs<R> na = m.nargs(h);
  PersistArgs pa = m.pargs();
  const float* zw = m.zw.p;
  void* args[] = {&sa, &na, &pa, &ncycles, &parity0, &zw};
  const PersistFn<R> fn = persist_fn<R>(h->tile_shell, m.uniform_npt == 5);
  Trace tr("persistent cycles");
  const cudaError_t e =
      cudaLaunchCooperativeKernel((const void*)fn, dim3(q.G), dim3(q.T), args, q.smem, h->stream);
  if (e == cudaErrorCooperativeLaunchTooLarge) {   // the wave no longer fits (another context holds SMs):
    cudaGetLastError();                             // the per-phase kernels take over for good
    q.on = false;
    return -1;
  }
  CK(e);
  h->launches++;
  return OR_OK;
}

template <class R>
int launch_cycle(or_ecycle* h, Impl<R>& m, int parity, cudaEvent_t* ev) {
  int rc;
  if (ev) CK(cudaEventRecord(ev[0], h->stream));
  // per-phase events need the kernels serialised
  const bool pdl = h->pdl && !ev;
  Trace tr(parity ? "cycle (odd)" : "cycle (even)");
  if ((rc = launch_loads<R>(h, m, parity))) return rc;     // FORCE (resol.F:2847), before the elements
  rc = h->tile_hex == 64 ? launch_hex<R, 64>(h, m, parity, pdl)
       : h->tile_hex == 128 ? launch_hex<R, 128>(h, m, parity, pdl) : launch_hex<R, 256>(h, m, parity, pdl);
  if (rc) return rc;
  if (ev) CK(cudaEventRecord(ev[1], h->stream));
  rc = h->tile_shell == 64 ? launch_shell_npt<R, 64>(h, m, parity, pdl)
       : h->tile_shell == 128 ? launch_shell_npt<R, 128>(h, m, parity, pdl)
                              : launch_shell_npt<R, 256>(h, m, parity, pdl);
  if (rc) return rc;
  if (ev) CK(cudaEventRecord(ev[2], h->stream));
  rc = launch_link<R>(h, m);
  if (rc) return rc;
  rc = launch_rbody<R>(h, m, parity);
  if (rc) return rc;
  rc = launch_node<R>(h, m, parity, pdl);
  if (rc) return rc;
  if (ev) CK(cudaEventRecord(ev[3], h->stream));
  return OR_OK;
}

template <class R>
int reset_impl(or_ecycle* h);

// NodeArgs::rotmask bits of part P's nodes, from its inertias and the rotational
// velocities vr (3 per node, part order): set where the part has rotations and the
// node's inertia or rotational velocity is nonzero, in the handle's precision.
template <class R>
void rot_bits(Impl<R>& m, const HPart& P, const double* vr) {
  for (int i = 0; i < P.numnod; ++i) {
    const int g = P.node_start + i;
    const bool on = P.has_rot && (R(P.in[i]) > R(0) || R(vr[3 * i]) != R(0) || R(vr[3 * i + 1]) != R(0) ||
                                  R(vr[3 * i + 2]) != R(0));
    unsigned& w = m.rotmask_h[g >> 5];
    w = on ? (w | (1u << (g & 31))) : (w & ~(1u << (g & 31)));
  }
}

template <class R>
int finalize_impl(or_ecycle* h) {
  typedef typename Vec4<R>::T R4;
  Impl<R>* mp = new Impl<R>();
  h->impl = mp;
  Impl<R>& m = *mp;
  m.nparts = (int)h->parts.size();
  // node layout
  int nn = 0, nt = 0;
  std::vector<int> tile_part;
  for (auto& P : h->parts) {
    P.node_start = nn;
    P.tile_start = nt;
    int pad = (P.numnod + NODE_TILE - 1) / NODE_TILE * NODE_TILE;
    P.node_pad = pad;
    for (int t = 0; t < pad / NODE_TILE; ++t) tile_part.push_back((int)(&P - &h->parts[0]));
    nn += pad;
    nt += pad / NODE_TILE;
    m.any_rot = m.any_rot || P.has_rot;
  }
  m.nnodpad = nn;
  m.ntiles = nt;
  // tiles left to the library (cfg.block_hex / block_shell 0): 64 elements per patch
  // when the patches at 64 fit one wave of the kernel's resident CTAs (a latency-bound
  // mesh gains from more CTAs), 128 otherwise; the autotuner times all three
  {
    auto tile_for = [&](long long nel, int ctas128) {
      return nel <= (long long)h->nsm * (2 * ctas128) * 64 ? 64 : 128;
    };
    long long nh = 0, ns = 0;
    for (auto& g : h->hex) nh += g.nel;
    for (auto& g : h->shell) ns += g.nel;
    if (h->cfg.block_hex == 0) h->tile_hex = tile_for(nh, Occupancy<R>::hex);
    if (h->cfg.block_shell == 0) h->tile_shell = tile_for(ns, Occupancy<R>::shell);
  }
  // patches
  std::vector<std::vector<std::pair<int, int>>> node_patch(nn);
  int rc = build_patches<8>(h, h->hex, h->tile_hex, m.hps, node_patch, 0);
  if (rc) return rc;
  const int nhp = (int)m.hps.info.size();
  rc = build_patches<4>(h, h->shell, h->tile_shell, m.sps, node_patch, nhp);
  if (rc) return rc;
  // load corners: their own slots, after every patch slot of their node (in load order)
  const int lbase = nhp + (int)m.sps.info.size();
  const int nload = (int)h->loads.size();
  std::vector<int> load_slot(4 * (size_t)nload, -1);
  for (int e = 0; e < nload; ++e) {
    const HLoad& L = h->loads[e];
    const int nc = L.type == 0 ? 1 : (L.node[3] >= 0 ? 4 : 3);
    for (int k = 0; k < nc; ++k)
      node_patch[h->parts[L.part].node_start + L.node[k]].push_back({lbase + 4 * e + k, 4 * e + k});
  }
  // node-major slots: per node, its (patch) entries in ascending patch number
  std::vector<int> adsky(nn + 1, 0);
  for (int n = 0; n < nn; ++n) adsky[n + 1] = adsky[n] + (int)node_patch[n].size();
  m.nslot = adsky[nn];
  for (int n = 0; n < nn; ++n) {
    auto& lst = node_patch[n];
    std::sort(lst.begin(), lst.end());
    for (size_t j = 0; j < lst.size(); ++j) {
      const int pid = lst[j].first, pos = lst[j].second;
      if (pid < nhp) m.hps.slots[pos] = adsky[n] + (int)j;
      else if (pid < lbase) m.sps.slots[pos] = adsky[n] + (int)j;
      else load_slot[pos] = adsky[n] + (int)j;
    }
  }
  node_patch.clear();
  node_patch.shrink_to_fit();
  // node arrays
  std::vector<double4> X(nn, make_double4(0, 0, 0, 0));
  std::vector<R4> V(nn, mk4(R(0), R(0), R(0), R(0))), VR(m.any_rot ? nn : 0, mk4(R(0), R(0), R(0), R(0)));
  std::vector<unsigned char> code(nn, 0);
  std::vector<PartDesc> pd;
  for (auto& P : h->parts) {
    for (int i = 0; i < P.numnod; ++i) {
      const int g = P.node_start + i;
      X[g] = make_double4(P.x[3 * i], P.x[3 * i + 1], P.x[3 * i + 2], (double)(R)P.ms[i]);
      V[g] = mk4(R(P.v[3 * i]), R(P.v[3 * i + 1]), R(P.v[3 * i + 2]), R(0));
      if (m.any_rot) VR[g] = mk4(R(P.vr[3 * i]), R(P.vr[3 * i + 1]), R(P.vr[3 * i + 2]), R(P.in[i]));
      code[g] = (unsigned char)((P.icodt[i] & 7) | ((P.icodr[i] & 7) << 3));
    }
    PartDesc d;
    d.node_start = P.node_start; d.node_end = P.node_start + P.numnod; d.tile_start = P.tile_start;
    d.has_rot = P.has_rot ? 1 : 0;
    pd.push_back(d);
  }
  // skewed /BCS: code bit 7 and the node's skew frame
  {
    std::vector<int> sof;
    for (auto& P : h->parts) {
      if (P.iskew.empty()) continue;
      for (int i = 0; i < P.numnod; ++i) {
        const int g = P.node_start + i;
        if (P.iskew[i] >= 0 && (P.icodt[i] | P.icodr[i])) {
          if (sof.empty()) sof.assign(nn, -1);
          sof[g] = P.iskew[i];
          code[g] |= 128;
        }
      }
    }
    std::vector<R> sk;
    for (auto& a : h->skews) for (int k = 0; k < 9; ++k) sk.push_back(R(a[k]));
    if ((rc = dput(h, m.skew_of, sof)) || (rc = dput(h, m.skw, sk))) return rc;
  }
  // loads and their time functions
  if (nload) {
    std::vector<LoadDesc> ld(nload);
    for (int e = 0; e < nload; ++e) {
      const HLoad& L = h->loads[e];
      LoadDesc d{};
      d.type = L.type; d.part = L.part; d.func = L.func; d.skew = L.skew; d.pad = 0;
      d.dir = L.type == 0 ? L.dir : (L.node[3] >= 0 ? 4 : 3);
      for (int k = 0; k < 4; ++k) {
        d.node[k] = L.node[k] >= 0 ? h->parts[L.part].node_start + L.node[k] : 0;
        d.slot[k] = load_slot[4 * (size_t)e + k];
      }
      d.fcx = L.fcx; d.fcy = L.fcy;
      ld[e] = d;
    }
    std::vector<FuncDesc> fd;
    std::vector<double> fxv, fyv;
    for (size_t f = 0; f < h->fx.size(); ++f) {
      fd.push_back(FuncDesc{(int)fxv.size(), (int)h->fx[f].size()});
      fxv.insert(fxv.end(), h->fx[f].begin(), h->fx[f].end());
      fyv.insert(fyv.end(), h->fy[f].begin(), h->fy[f].end());
    }
    m.nload = nload;
    std::vector<double> zl(nload, 0.0);
    if ((rc = dput(h, m.loadd, ld)) || (rc = dput(h, m.funcd, fd)) || (rc = dput(h, m.funcx, fxv)) ||
        (rc = dput(h, m.funcy, fyv)) || (rc = dput(h, m.wacc, zl)) || (rc = dput(h, m.wpend, zl)))
      return rc;
  }
  // rigid links: node lists in global padded numbering, code bit 6 on their nodes
  if (!h->links.empty()) {
    std::vector<LinkDesc> ld;
    std::vector<int> ln, lof(nn, -1);
    for (auto& L : h->links) {
      LinkDesc d;
      d.first = (int)ln.size(); d.count = (int)L.nodes.size(); d.ic = L.ic; d.icr = L.icr;
      const int base = h->parts[L.part].node_start;
      for (int n : L.nodes) {
        ln.push_back(base + n);
        lof[base + n] = (int)ld.size();
        code[base + n] |= 64;
      }
      ld.push_back(d);
    }
    m.nlinks = (int)ld.size();
    if ((rc = dput(h, m.linkd, ld)) || (rc = dput(h, m.link_nodes, ln)) || (rc = dput(h, m.link_of, lof)) ||
        (rc = dalloc(h, m.link_mean, ld.size())))
      return rc;
    CK(cudaMemset(m.link_mean.p, 0, m.link_mean.n * sizeof(LinkMean)));
  }
  // rigid bodies: descriptors in add order, secondary nodes in global padded numbering
  if (!h->rbodies.empty()) {
    std::vector<RBodyDesc> bd;
    std::vector<int> sl;
    std::vector<unsigned char> role(nn, 0);
    for (auto& B : h->rbodies) {
      const int base = h->parts[B.part].node_start;
      RBodyDesc d;
      d.master = base + B.master; d.first = (int)sl.size(); d.count = (int)B.slaves.size(); d.part = B.part;
      if (code[d.master] & 64) return fail(h, OR_E_UNSUPPORTED, "rigid body node in a rigid link");
      role[d.master] = 1;
      for (int n : B.slaves) {
        if (code[base + n] & 64) return fail(h, OR_E_UNSUPPORTED, "rigid body node in a rigid link");
        sl.push_back(base + n);
        role[base + n] = 2;
      }
      bd.push_back(d);
      for (int k = 0; k < 12; ++k) m.rby0.push_back(R(B.rby[k]));
    }
    m.nrb = (int)bd.size();
    if ((rc = dput(h, m.rbd, bd)) || (rc = dput(h, m.rb_nodes, sl)) || (rc = dput(h, m.rby, m.rby0)) ||
        (rc = dput(h, m.rb_role, role)) || (rc = dput(h, m.rb_ek, std::vector<double>(m.nrb, 0.0))) ||
        (rc = dput(h, m.rb_ekr, std::vector<double>(m.nrb, 0.0))))
      return rc;
  }
  if (m.any_rot) {
    m.rotmask_h.assign((nn + 31) / 32, 0u);
    for (auto& P : h->parts)
      if (P.has_rot) rot_bits<R>(m, P, P.vr.data());
    long long nrot = 0;
    for (unsigned w : m.rotmask_h) nrot += __builtin_popcount(w);
    m.rot_sparse = 2 * nrot < (long long)nn ? 1 : 0;
  }
  if ((rc = dput(h, m.X, X)) || (rc = dput(h, m.V, V)) || (rc = dput(h, m.VR, VR)) || (rc = dput(h, m.code, code)) ||
      (rc = dput(h, m.adsky, adsky)) || (rc = dput(h, m.tile_part, tile_part)) || (rc = dput(h, m.partd, pd)) ||
      (rc = dput(h, m.rotmask, m.rotmask_h)))
    return rc;
  std::vector<double> zero(nn, 0.0);
  if ((rc = dput(h, m.DX, zero)) || (rc = dput(h, m.DY, zero)) || (rc = dput(h, m.DZ, zero))) return rc;
  {
    int maxn = 0;
    for (auto& P : h->parts) maxn = std::max(maxn, P.numnod);
    if ((rc = dalloc(h, m.stage, 3 * (size_t)maxn))) return rc;
  }
  if ((rc = dalloc(h, m.fslot, (size_t)m.nslot))) return rc;
  CK(cudaMemset(m.fslot.p, 0, m.fslot.n * sizeof(R4)));
  if (!h->shell.empty()) {
    if ((rc = dalloc(h, m.mslot, (size_t)m.nslot))) return rc;
    CK(cudaMemset(m.mslot.p, 0, m.mslot.n * sizeof(R4)));
  }
  if ((rc = dalloc(h, m.time, 2 * (size_t)m.nparts)) || (rc = dalloc(h, m.acc, 2 * (size_t)m.nparts)) ||
      (rc = dalloc(h, m.err, 1)))
    return rc;
  CK(cudaMemset(m.err.p, 0, sizeof(ErrorWord)));
  if ((rc = dput(h, m.ekin, std::vector<double>(m.ntiles, 0.0))) || (rc = dput(h, m.ekinr, std::vector<double>(m.ntiles, 0.0))))
    return rc;
  // hexas
  if (!h->hex.empty()) {
    PatchSet& ps = m.hps;
    const int np = ps.nelpad;
    std::vector<HexGroupDesc> desc;
    for (auto& g : h->hex) {
      HexGroupDesc d{};
      d.part = g.part; d.law = g.mat.law; d.nel = g.nel; d.jcvt = g.prop.jcvt;
      m.any_corot = m.any_corot || g.prop.jcvt != 0;
      d.rho0 = g.mat.rho0; d.shear = g.mat.shear; d.bulk = g.mat.bulk; d.jc_a = g.mat.jc_a; d.jc_b = g.mat.jc_b;
      d.jc_n = g.mat.jc_n; d.epsmax = g.mat.epsmax; d.sigmax = g.mat.sigmax;
      d.qa = g.prop.qa; d.qb = g.prop.qb; d.qh = g.prop.qh; d.dtfac = h->cfg.dtfac_solid; d.dtmin = h->cfg.dtmin_solid;
      desc.push_back(d);
    }
    std::vector<uint4> conn(np, make_uint4(0, 0, 0, 0));
    std::vector<int> elem(np, 0);
    std::vector<R> rho(np, R(0)), vol0(np, R(0));
    std::vector<double> vol0dp(np, 0.0);
    for (int ie = 0; ie < np; ++ie) {
      const int gi = ps.elem_group[ie];
      if (gi < 0) continue;
      const uint16_t* l = &ps.local[(size_t)ie * 8];
      conn[ie] = make_uint4(l[0] | (unsigned)l[1] << 16, l[2] | (unsigned)l[3] << 16, l[4] | (unsigned)l[5] << 16,
                            l[6] | (unsigned)l[7] << 16);
      const HHex& g = h->hex[gi];
      const int ue = ps.elem_user[ie];
      elem[ie] = g.gofs + ue;
      rho[ie] = R(g.mat.rho0);
      vol0[ie] = R(g.vol0[ue]);
      vol0dp[ie] = g.vol0[ue];
    }
    std::vector<int> pn, pslot;
    padded_lists(ps, pn, pslot);
    std::vector<uint16_t> inc;
    incidence_lists(ps, 8, h->tile_hex, inc);
    m.hinc_stride = incidence_stride(ps, 8, h->tile_hex);
    if ((rc = dput(h, m.hinc, inc))) return rc;
    if ((rc = dput(h, m.hpatch, ps.info)) || (rc = dput(h, m.hdesc, desc)) || (rc = dput(h, m.hnodes, pn)) ||
        (rc = dput(h, m.hslots, pslot)) || (rc = dput(h, m.helem, elem)) || (rc = dput(h, m.hconn, conn)) ||
        (rc = dput(h, m.hrho, rho)) || (rc = dput(h, m.hvol0, vol0)) || (rc = dput(h, m.hvol0dp, vol0dp)))
      return rc;
    std::vector<R> z(np, R(0));
    if ((rc = dput(h, m.heint, z)) || (rc = dput(h, m.hqvis, z)) || (rc = dput(h, m.hpla, z)) || (rc = dput(h, m.hepsd, z)))
      return rc;
    if ((rc = dalloc(h, m.hsig, 6 * (size_t)np))) return rc;
    CK(cudaMemset(m.hsig.p, 0, m.hsig.n * sizeof(R)));
    if ((rc = dput(h, m.hehour, std::vector<double>(ps.info.size(), 0.0))) ||
        (rc = dput(h, m.hwpla, std::vector<double>(ps.info.size(), 0.0))))
      return rc;
  }
  // shells
  if (!h->shell.empty()) {
    PatchSet& ps = m.sps;
    const int np = ps.nelpad;
    std::vector<ShellGroupDesc> desc;
    bool any_jca = false;
    for (auto& g : h->shell) {
      ShellGroupDesc d{};
      d.part = g.part; d.law = g.mat.law; d.nel = g.nel; d.npt = g.prop.npt; d.ithk = g.prop.ithk;
      d.ishfram = g.prop.ishfram;
      d.ipla = g.prop.ipla;
      d.ihbe = shell_ihbe(g.prop.ishell, g.prop.npt);
      d.dn = g.prop.dn;
      d.has_jca = g.jca.empty() ? 0 : 1;
      any_jca = any_jca || !g.jca.empty();
      d.rho0 = g.mat.rho0; d.young = g.mat.young; d.nu = g.mat.nu; d.shear = g.mat.shear; d.a11 = g.mat.a11;
      d.a12 = g.mat.a12; d.ssp = g.mat.ssp_shell; d.jc_a = g.mat.jc_a; d.jc_b = g.mat.jc_b; d.jc_n = g.mat.jc_n;
      d.sigmax = g.mat.sigmax; d.hm = g.prop.hm; d.hf = g.prop.hf; d.hr = g.prop.hr; d.shf = g.prop.shf;
      d.pressure = g.prop.pressure; d.dtfac = h->cfg.dtfac_shell; d.dtmin = h->cfg.dtmin_shell;
      desc.push_back(d);
      m.maxnpt = std::max(m.maxnpt, g.prop.npt);
    }
    m.uniform_npt = h->shell[0].prop.npt == 5 ? 5 : 0;
    for (auto& g : h->shell)
      if (g.prop.npt != 5 || shell_ihbe(g.prop.ishell, g.prop.npt) != 1 || g.prop.ipla != 0) m.uniform_npt = 0;
    std::vector<uint2> conn(np, make_uint2(0, 0));
    std::vector<int> elem(np, 0), degen(np, 0);
    std::vector<R> thke(np, R(1)), jca(any_jca ? np : 0, R(0));
    for (int ie = 0; ie < np; ++ie) {
      const int gi = ps.elem_group[ie];
      if (gi < 0) continue;
      const uint16_t* l = &ps.local[(size_t)ie * 4];
      conn[ie] = make_uint2(l[0] | (unsigned)l[1] << 16, l[2] | (unsigned)l[3] << 16);
      const HShell& g = h->shell[gi];
      const int ue = ps.elem_user[ie];
      elem[ie] = g.gofs + ue;
      degen[ie] = g.conn[4 * (size_t)ue + 2] == g.conn[4 * (size_t)ue + 3] ? 1 : 0;
      thke[ie] = R(g.thke[ue]);
      if (any_jca) jca[ie] = R(g.jca.empty() ? g.mat.jc_a : g.jca[ue]);
    }
    std::vector<int> pn, pslot;
    padded_lists(ps, pn, pslot);
    std::vector<uint16_t> inc;
    incidence_lists(ps, 4, h->tile_shell, inc);
    m.sinc_stride = incidence_stride(ps, 4, h->tile_shell);
    if ((rc = dput(h, m.sinc, inc))) return rc;
    if ((rc = dput(h, m.spatch, ps.info)) || (rc = dput(h, m.sdesc, desc)) || (rc = dput(h, m.snodes, pn)) ||
        (rc = dput(h, m.sslots, pslot)) || (rc = dput(h, m.selem, elem)) || (rc = dput(h, m.sdegen, degen)) ||
        (rc = dput(h, m.sconn, conn)) || (rc = dput(h, m.sthke, thke)) || (rc = dput(h, m.sthk, thke)) ||
        (rc = dput(h, m.sjca, jca)))
      return rc;
    if ((rc = dalloc(h, m.ssig, (size_t)m.maxnpt * 5 * np)) || (rc = dalloc(h, m.spla, (size_t)m.maxnpt * np)) ||
        (rc = dalloc(h, m.shourg, 3 * (size_t)np)) || (rc = dalloc(h, m.seint, 2 * (size_t)np)))
      return rc;
    CK(cudaMemset(m.ssig.p, 0, m.ssig.n * sizeof(R)));
    CK(cudaMemset(m.spla.p, 0, m.spla.n * sizeof(R)));
    CK(cudaMemset(m.shourg.p, 0, m.shourg.n * sizeof(R)));
    CK(cudaMemset(m.seint.p, 0, m.seint.n * sizeof(R)));
    std::vector<float> zw(&ZW_TABLE[0][0], &ZW_TABLE[0][0] + 10 * 33);
    if ((rc = dput(h, m.zw, zw))) return rc;
    if ((rc = dput(h, m.sehour, std::vector<double>(ps.info.size(), 0.0))) ||
        (rc = dput(h, m.swpla, std::vector<double>(ps.info.size(), 0.0))))
      return rc;
  }
  rc = set_smem_attrs<R>(h, m);
  if (rc) return rc;
  if ((rc = persist_build<R>(h, m))) return rc;
  CK(cudaDeviceSynchronize());
  return OR_OK;
}

// Re-uploads the initial node arrays and re-initialises the element state.
template <class R>
int reset_impl(or_ecycle* h) {
  typedef typename Vec4<R>::T R4;
  Impl<R>& m = *(Impl<R>*)h->impl;
  const int nn = m.nnodpad;
  CK(cudaStreamSynchronize(h->stream));
  std::vector<double4> X(nn, make_double4(0, 0, 0, 0));
  std::vector<R4> V(nn, mk4(R(0), R(0), R(0), R(0))), VR(m.any_rot ? nn : 0, mk4(R(0), R(0), R(0), R(0)));
  for (auto& P : h->parts)
    for (int i = 0; i < P.numnod; ++i) {
      const int g = P.node_start + i;
      X[g] = make_double4(P.x[3 * i], P.x[3 * i + 1], P.x[3 * i + 2], (double)(R)P.ms[i]);
      V[g] = mk4(R(P.v[3 * i]), R(P.v[3 * i + 1]), R(P.v[3 * i + 2]), R(0));
      if (m.any_rot) VR[g] = mk4(R(P.vr[3 * i]), R(P.vr[3 * i + 1]), R(P.vr[3 * i + 2]), R(P.in[i]));
    }
  CK(cudaMemcpy(m.X.p, X.data(), X.size() * sizeof(double4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m.V.p, V.data(), V.size() * sizeof(R4), cudaMemcpyHostToDevice));
  if (m.any_rot) {
    CK(cudaMemcpy(m.VR.p, VR.data(), VR.size() * sizeof(R4), cudaMemcpyHostToDevice));
    for (auto& P : h->parts)
      if (P.has_rot) rot_bits<R>(m, P, P.vr.data());
    CK(cudaMemcpy(m.rotmask.p, m.rotmask_h.data(), m.rotmask_h.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
  }
  CK(cudaMemset(m.DX.p, 0, nn * sizeof(double)));
  CK(cudaMemset(m.DY.p, 0, nn * sizeof(double)));
  CK(cudaMemset(m.DZ.p, 0, nn * sizeof(double)));
  if (m.nload) {
    CK(cudaMemset(m.wacc.p, 0, m.wacc.n * sizeof(double)));
    CK(cudaMemset(m.wpend.p, 0, m.wpend.n * sizeof(double)));
  }
  if (!h->hex.empty()) {
    const int np = m.hps.nelpad;
    std::vector<R> rho(np, R(0));
    for (int ie = 0; ie < np; ++ie) {
      const int gi = m.hps.elem_group[ie];
      if (gi >= 0) rho[ie] = R(h->hex[gi].mat.rho0);
    }
    CK(cudaMemcpy(m.hrho.p, rho.data(), np * sizeof(R), cudaMemcpyHostToDevice));
    CK(cudaMemset(m.heint.p, 0, np * sizeof(R)));
    CK(cudaMemset(m.hqvis.p, 0, np * sizeof(R)));
    CK(cudaMemset(m.hpla.p, 0, np * sizeof(R)));
    CK(cudaMemset(m.hepsd.p, 0, np * sizeof(R)));
    CK(cudaMemset(m.hsig.p, 0, m.hsig.n * sizeof(R)));
    CK(cudaMemset(m.hehour.p, 0, m.hehour.n * sizeof(double)));
    CK(cudaMemset(m.hwpla.p, 0, m.hwpla.n * sizeof(double)));
  }
  if (!h->shell.empty()) {
    CK(cudaMemcpy(m.sthk.p, m.sthke.p, m.sthk.n * sizeof(R), cudaMemcpyDeviceToDevice));
    CK(cudaMemset(m.ssig.p, 0, m.ssig.n * sizeof(R)));
    CK(cudaMemset(m.spla.p, 0, m.spla.n * sizeof(R)));
    CK(cudaMemset(m.shourg.p, 0, m.shourg.n * sizeof(R)));
    CK(cudaMemset(m.seint.p, 0, m.seint.n * sizeof(R)));
    CK(cudaMemset(m.sehour.p, 0, m.sehour.n * sizeof(double)));
    CK(cudaMemset(m.swpla.p, 0, m.swpla.n * sizeof(double)));
  }
  CK(cudaMemset(m.ekin.p, 0, m.ekin.n * sizeof(double)));
  CK(cudaMemset(m.ekinr.p, 0, m.ekinr.n * sizeof(double)));
  if (m.nrb) {
    CK(cudaMemcpy(m.rby.p, m.rby0.data(), m.rby0.size() * sizeof(R), cudaMemcpyHostToDevice));
    CK(cudaMemset(m.rb_ek.p, 0, m.rb_ek.n * sizeof(double)));
    CK(cudaMemset(m.rb_ekr.p, 0, m.rb_ekr.n * sizeof(double)));
  }
  CK(cudaDeviceSynchronize());
  return OR_OK;
}

int wait_stream(or_ecycle* h, cudaEvent_t ev) {
  double limit = 900.0;
  if (const char* s = std::getenv("OR_ECYCLE_TIMEOUT_S")) limit = std::atof(s);
  auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t q = cudaEventQuery(ev);
    if (q == cudaSuccess) return OR_OK;
    if (q != cudaErrorNotReady) return fail(h, OR_E_CUDA, std::string("stream: ") + cudaGetErrorString(q));
    double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > limit) return fail(h, OR_E_TIMEOUT, "bounded wait expired");
    std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 5 : 200));
  }
}

// Bounded wait for everything queued on the handle's stream so far.  Callers
// read results back only after it: a copy into pageable host memory blocks until
// the stream drains, so issued first it would make the wait unbounded.  On
// OR_E_TIMEOUT the work keeps running and the event is left to it.
int wait_queued(or_ecycle* h) {
  cudaEvent_t ev;
  CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ev, h->stream));
  const int rc = wait_stream(h, ev);
  if (rc == OR_E_TIMEOUT) return rc;
  cudaEventDestroy(ev);
  return rc;
}

template <class R>
int step_impl(or_ecycle* h, int ncycles, or_ecycle_time* t) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const int np = m.nparts;
  std::vector<PartTime> pt(np);
  for (int p = 0; p < np; ++p) {
    pt[p].tt = t[p].tt; pt[p].dt2 = t[p].dt2; pt[p].dt2old = t[p].dt2old; pt[p].dt1 = t[p].dt1;
    pt[p].dt12 = t[p].dt12; pt[p].ncycle = t[p].ncycle; pt[p].ityptst = t[p].ityptst; pt[p].neltst = t[p].neltst;
    pt[p].pad = 0;
  }
  std::vector<PartAcc> acc0(np);
  for (auto& a : acc0) { a.dtkey = ~0ull; a.dtbits = ~0ull; }
  h->launches = 0;
  CK(cudaMemcpyAsync(m.time.p, pt.data(), np * sizeof(PartTime), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(m.acc.p, acc0.data(), np * sizeof(PartAcc), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemsetAsync(m.err.p, 0, sizeof(ErrorWord), h->stream));
  int rc;
  const bool use_graph = h->cfg.graph != 0;
  int done = 0;
  if (m.per.on) {            // every cycle in cooperative launches of an even number of cycles
    constexpr int CHUNK = 1 << 20;
    while (done < ncycles) {
      const int nc = std::min(CHUNK, ncycles - done);
      rc = launch_persistent<R>(h, m, nc, done & 1);
      if (rc < 0) break;       // fell back: the remaining cycles run below
      if (rc) return rc;
      done += nc;
    }
  }
  if (use_graph && ncycles - done >= GRAPH_CYCLES) {
    if (!h->graph_exec) {
      CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      long long l0 = h->launches;
      for (int c = 0; c < GRAPH_CYCLES; ++c) {
        rc = launch_cycle<R>(h, m, c & 1, nullptr);
        if (rc) { cudaGraph_t g; cudaStreamEndCapture(h->stream, &g); if (g) cudaGraphDestroy(g); return rc; }
      }
      CK(cudaStreamEndCapture(h->stream, &h->graph));
      CK(cudaGraphInstantiate(&h->graph_exec, h->graph, 0));
      h->graph_launches = h->launches - l0;      // kernels in one replay (loads and links included)
      h->launches = l0;
    }
    for (; done + GRAPH_CYCLES <= ncycles; done += GRAPH_CYCLES) {
      CK(cudaGraphLaunch(h->graph_exec, h->stream));
      h->launches += h->graph_launches;
    }
  }
  // eager cycles; without a graph each phase is bracketed by events, read back
  // once per chunk of cycles so that the host keeps the launch queue full
  constexpr int TCHUNK = 64;
  const bool timing = !use_graph;
  std::vector<cudaEvent_t> ev;
  if (timing) {
    ev.resize(4 * (size_t)std::min(TCHUNK, std::max(1, ncycles - done)));
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (double& x : h->phase_ms) x = 0;
  }
  while (done < ncycles) {
    const int nc = timing ? std::min(TCHUNK, ncycles - done) : ncycles - done;
    for (int c = 0; c < nc; ++c) {
      rc = launch_cycle<R>(h, m, (done + c) & 1, timing ? &ev[4 * (size_t)c] : nullptr);
      if (rc) return rc;
    }
    if (timing) {
      CK(cudaEventSynchronize(ev[4 * (size_t)(nc - 1) + 3]));
      for (int c = 0; c < nc; ++c) {
        float a, b, d;
        cudaEventElapsedTime(&a, ev[4 * c], ev[4 * c + 1]);
        cudaEventElapsedTime(&b, ev[4 * c + 1], ev[4 * c + 2]);
        cudaEventElapsedTime(&d, ev[4 * c + 2], ev[4 * c + 3]);
        h->phase_ms[0] += a; h->phase_ms[1] += b; h->phase_ms[2] += d; h->phase_ms[3] += a + b + d;
      }
    }
    done += nc;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  const int fin = ncycles & 1;
  h->next_parity = fin;
  if ((rc = wait_queued(h))) return rc;
  CK(cudaMemcpyAsync(pt.data(), m.time.p + fin * np, np * sizeof(PartTime), cudaMemcpyDeviceToHost, h->stream));
  ErrorWord ew{};
  CK(cudaMemcpyAsync(&ew, m.err.p, sizeof(ErrorWord), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int p = 0; p < np; ++p) {
    t[p].tt = pt[p].tt; t[p].dt1 = pt[p].dt1; t[p].dt2 = pt[p].dt2; t[p].dt12 = pt[p].dt12;
    t[p].dt2old = pt[p].dt2old; t[p].ncycle = pt[p].ncycle; t[p].ityptst = pt[p].ityptst; t[p].neltst = pt[p].neltst;
  }
  h->last_code = ew.code;
  h->last_index = ew.index;
  if (ew.code) {
    char buf[160];
    snprintf(buf, sizeof buf, "device error %d at index %d", ew.code, ew.index);
    return fail(h, ew.code, buf);
  }
  return OR_OK;
}

// Device time of one launch of each phase kernel: `reps` launches of the same
// kernel captured back to back in a graph, replayed once between two events
// on the handle's stream.  The repeated launches advance the state, which is
// then reset to the uploaded one.
template <class R>
int kernel_times_impl(or_ecycle* h, int reps, double* us) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const int parity = h->next_parity;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int rc = OR_OK;
  for (int ph = 0; ph < 3 && rc == OR_OK; ++ph) {
    us[ph] = 0.0;
    if ((ph == 0 && m.hps.info.empty()) || (ph == 1 && m.sps.info.empty())) continue;
    auto launch = [&]() -> int {
      if (ph == 0)
        return h->tile_hex == 64 ? launch_hex<R, 64>(h, m, parity)
               : h->tile_hex == 128 ? launch_hex<R, 128>(h, m, parity) : launch_hex<R, 256>(h, m, parity);
      if (ph == 1)
        return h->tile_shell == 64 ? launch_shell_npt<R, 64>(h, m, parity)
               : h->tile_shell == 128 ? launch_shell_npt<R, 128>(h, m, parity) : launch_shell_npt<R, 256>(h, m, parity);
      return launch_node<R>(h, m, parity);
    };
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < reps && rc == OR_OK; ++i) rc = launch();
    cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
    if (rc == OR_OK && ec != cudaSuccess) rc = fail(h, OR_E_CUDA, cudaGetErrorString(ec));
    if (rc == OR_OK && (ec = cudaGraphInstantiate(&ge, g, 0)) != cudaSuccess) rc = fail(h, OR_E_CUDA, cudaGetErrorString(ec));
    if (rc == OR_OK) {
      float ms = 0.f;
      if (cudaGraphLaunch(ge, h->stream) != cudaSuccess || cudaEventRecord(e0, h->stream) != cudaSuccess ||
          cudaGraphLaunch(ge, h->stream) != cudaSuccess || cudaEventRecord(e1, h->stream) != cudaSuccess ||
          cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
        rc = fail(h, OR_E_CUDA, "kernel timing replay");
      us[ph] = 1e3 * (double)ms / reps;
    }
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  h->next_parity = 0;
  return reset_impl<R>(h);
}

template <class R>
int get_nodes_impl(or_ecycle* h, int part, double* x, double* d, double* v, double* vr) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const HPart& P = h->parts[part];
  const int n = P.numnod, s = P.node_start;
  if (n == 0) return OR_OK;
  if (vr && !m.VR.p) std::fill(vr, vr + 3 * (size_t)n, 0.0);
  double* dst[4] = {x, d, v, m.VR.p ? vr : nullptr};
  for (int kind = 0; kind < 4; ++kind) {
    if (!dst[kind]) continue;
    node_io_kernel<R><<<(n + 255) / 256, 256, 0, h->stream>>>(kind, 0, m.stage.p, n, s, m.X.p, m.DX.p, m.DY.p, m.DZ.p,
                                                             m.V.p, m.VR.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst[kind], m.stage.p, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return OR_OK;
}

template <class R>
int set_nodes_impl(or_ecycle* h, int part, const double* x, const double* d, const double* v, const double* vr) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const HPart& P = h->parts[part];
  const int n = P.numnod, s = P.node_start;
  if (n == 0) return OR_OK;
  const double* src[4] = {x, d, v, m.VR.p ? vr : nullptr};
  for (int kind = 0; kind < 4; ++kind) {
    if (!src[kind]) continue;
    // copy the caller's array (DMA when it is pinned), then scatter it on the device;
    // stream order keeps the staging buffer free until the kernel has read it
    CK(cudaMemcpyAsync(m.stage.p, src[kind], 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    node_io_kernel<R><<<(n + 255) / 256, 256, 0, h->stream>>>(kind, 1, m.stage.p, n, s, m.X.p, m.DX.p, m.DY.p, m.DZ.p,
                                                             m.V.p, m.VR.p);
    CK(cudaGetLastError());
  }
  if (src[3] && P.has_rot) {     // a rotational velocity set on a node without inertia
    rot_bits<R>(m, P, vr);
    CK(cudaMemcpyAsync(m.rotmask.p, m.rotmask_h.data(), m.rotmask_h.size() * sizeof(unsigned), cudaMemcpyHostToDevice,
                       h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return OR_OK;
}

template <class R>
std::vector<R> d2h(const R* p, size_t n) {
  std::vector<R> v(n);
  if (n) cudaMemcpy(v.data(), p, n * sizeof(R), cudaMemcpyDeviceToHost);
  return v;
}

template <class R>
int hex_state_impl(or_ecycle* h, int gi, double* sig, double* eint, double* rho, double* qvis, double* pla, double* epsd) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const HHex& g = h->hex[gi];
  const int np = m.hps.nelpad;
  CK(cudaStreamSynchronize(h->stream));
  if (sig) {
    auto s = d2h(m.hsig.p, 6 * (size_t)np);
    for (int c = 0; c < 6; ++c)
      for (int i = 0; i < g.nel; ++i) sig[(size_t)c * g.nel + i] = s[(size_t)c * np + g.internal[i]];
  }
  auto one = [&](double* out, const DBuf<R>& b) {
    if (!out) return;
    auto s = d2h(b.p, (size_t)np);
    for (int i = 0; i < g.nel; ++i) out[i] = s[g.internal[i]];
  };
  one(eint, m.heint); one(rho, m.hrho); one(qvis, m.hqvis); one(pla, m.hpla); one(epsd, m.hepsd);
  CK(cudaGetLastError());
  return OR_OK;
}

template <class R>
int shell_state_impl(or_ecycle* h, int gi, double* sig, double* pla, double* thk, double* hourg, double* eint) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const HShell& g = h->shell[gi];
  const int np = m.sps.nelpad, npt = g.prop.npt;
  CK(cudaStreamSynchronize(h->stream));
  if (sig) {
    auto s = d2h(m.ssig.p, m.ssig.n);
    for (int q = 0; q < npt * 5; ++q)
      for (int i = 0; i < g.nel; ++i) sig[(size_t)q * g.nel + i] = s[(size_t)q * np + g.internal[i]];
  }
  if (pla) {
    auto s = d2h(m.spla.p, m.spla.n);
    for (int q = 0; q < npt; ++q)
      for (int i = 0; i < g.nel; ++i) pla[(size_t)q * g.nel + i] = s[(size_t)q * np + g.internal[i]];
  }
  if (thk) {
    auto s = d2h(m.sthk.p, (size_t)np);
    for (int i = 0; i < g.nel; ++i) thk[i] = s[g.internal[i]];
  }
  if (hourg) {
    auto s = d2h(m.shourg.p, 3 * (size_t)np);
    for (int q = 0; q < 3; ++q)
      for (int i = 0; i < g.nel; ++i) hourg[(size_t)q * g.nel + i] = s[(size_t)q * np + g.internal[i]];
  }
  if (eint) {
    auto s = d2h(m.seint.p, 2 * (size_t)np);
    for (int q = 0; q < 2; ++q)
      for (int i = 0; i < g.nel; ++i) eint[(size_t)q * g.nel + i] = s[(size_t)q * np + g.internal[i]];
  }
  CK(cudaGetLastError());
  return OR_OK;
}

// element state upload (restart): the group's elements at their internal indices
template <class R>
int put_group(or_ecycle* h, R* dev, size_t np, int ncomp, const std::vector<int>& internal, const double* src) {
  if (!src) return OR_OK;
  auto s = d2h(dev, (size_t)ncomp * np);
  const size_t nel = internal.size();
  for (int q = 0; q < ncomp; ++q)
    for (size_t i = 0; i < nel; ++i) s[(size_t)q * np + internal[i]] = R(src[(size_t)q * nel + i]);
  CK(cudaMemcpy(dev, s.data(), s.size() * sizeof(R), cudaMemcpyHostToDevice));
  return OR_OK;
}

template <class R>
int set_hex_state_impl(or_ecycle* h, int gi, const double* sig, const double* eint, const double* rho,
                       const double* qvis, const double* pla, const double* epsd) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const HHex& g = h->hex[gi];
  const size_t np = m.hps.nelpad;
  CK(cudaStreamSynchronize(h->stream));
  int rc;
  if ((rc = put_group(h, m.hsig.p, np, 6, g.internal, sig)) || (rc = put_group(h, m.heint.p, np, 1, g.internal, eint)) ||
      (rc = put_group(h, m.hrho.p, np, 1, g.internal, rho)) || (rc = put_group(h, m.hqvis.p, np, 1, g.internal, qvis)) ||
      (rc = put_group(h, m.hpla.p, np, 1, g.internal, pla)) || (rc = put_group(h, m.hepsd.p, np, 1, g.internal, epsd)))
    return rc;
  return OR_OK;
}

template <class R>
int set_shell_state_impl(or_ecycle* h, int gi, const double* sig, const double* pla, const double* thk,
                         const double* hourg, const double* eint) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const HShell& g = h->shell[gi];
  const size_t np = m.sps.nelpad;
  const int npt = g.prop.npt;
  CK(cudaStreamSynchronize(h->stream));
  int rc;
  if ((rc = put_group(h, m.ssig.p, np, 5 * npt, g.internal, sig)) || (rc = put_group(h, m.spla.p, np, npt, g.internal, pla)) ||
      (rc = put_group(h, m.sthk.p, np, 1, g.internal, thk)) || (rc = put_group(h, m.shourg.p, np, 3, g.internal, hourg)) ||
      (rc = put_group(h, m.seint.p, np, 2, g.internal, eint)))
    return rc;
  return OR_OK;
}

template <class R>
int energies_impl(or_ecycle* h, int part, or_energies* e) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  CK(cudaStreamSynchronize(h->stream));
  double ei = 0, eh = 0, wp = 0, ek = 0, ekr = 0;
  if (!h->hex.empty()) {
    auto eint = d2h(m.heint.p, m.heint.n);
    auto vol0 = d2h(m.hvol0.p, m.hvol0.n);
    auto ehour = d2h(m.hehour.p, m.hehour.n);
    auto wpla = d2h(m.hwpla.p, m.hwpla.n);
    for (size_t ie = 0; ie < eint.size(); ++ie) {
      const int gi = m.hps.elem_group[ie];
      if (gi >= 0 && h->hex[gi].part == part) ei += (double)eint[ie] * (double)vol0[ie];
    }
    for (size_t p = 0; p < m.hps.info.size(); ++p)
      if (h->hex[m.hps.info[p].group].part == part) { eh += ehour[p]; wp += wpla[p]; }
  }
  if (!h->shell.empty()) {
    auto eint = d2h(m.seint.p, m.seint.n);
    auto ehour = d2h(m.sehour.p, m.sehour.n);
    auto wpla = d2h(m.swpla.p, m.swpla.n);
    const size_t np = m.sps.nelpad;
    for (size_t ie = 0; ie < np; ++ie) {
      const int gi = m.sps.elem_group[ie];
      if (gi >= 0 && h->shell[gi].part == part) ei += (double)eint[ie] + (double)eint[np + ie];
    }
    for (size_t p = 0; p < m.sps.info.size(); ++p)
      if (h->shell[m.sps.info[p].group].part == part) { eh += ehour[p]; wp += wpla[p]; }
  }
  auto ekin = d2h(m.ekin.p, m.ekin.n);
  auto ekinr = d2h(m.ekinr.p, m.ekinr.n);
  const HPart& P = h->parts[part];
  for (int t = P.tile_start; t < P.tile_start + P.node_pad / NODE_TILE; ++t) { ek += ekin[t]; ekr += ekinr[t]; }
  if (m.nrb) {      // the bodies' energies (their nodes are left out of the tiles), in add order
    auto bk = d2h(m.rb_ek.p, m.rb_ek.n);
    auto bkr = d2h(m.rb_ekr.p, m.rb_ekr.n);
    for (int b = 0; b < m.nrb; ++b)
      if (h->rbodies[b].part == part) { ek += bk[b]; ekr += bkr[b]; }
  }
  // external work of the part's loads: the cumulative sums, plus the last cycle's
  // concentrated-load power times that cycle's DT2
  double wx = 0.0;
  if (m.nload) {
    auto wacc = d2h(m.wacc.p, m.wacc.n);
    auto wpend = d2h(m.wpend.p, m.wpend.n);
    PartTime t{};
    CK(cudaMemcpy(&t, m.time.p + h->next_parity * m.nparts + part, sizeof(PartTime), cudaMemcpyDeviceToHost));
    for (int e = 0; e < m.nload; ++e)
      if (h->loads[e].part == part) wx += wacc[e] + wpend[e] * t.dt2;
  }
  e->internal = ei; e->kinetic = ek; e->kinetic_rot = ekr;
  e->hourglass = P.ehour0 + eh; e->plastic_work = P.wpla0 + wp; e->external_work = P.wext0 + wx;
  CK(cudaGetLastError());
  return OR_OK;
}

template <class R>
void destroy_impl(or_ecycle* h) {
  if (!h->impl) return;
  Impl<R>* m = (Impl<R>*)h->impl;
  m->free_all();
  delete m;
  h->impl = nullptr;
}

// ----------------------------------------------------------------------------
// domain decomposition: one part split over ranks, one boundary-force exchange
// and one time-step minimum per cycle (the reference's SPMD_EXCH_A and
// SPMD_GLOB_MIN5), the exchange itself left to the caller (NCCL, gloo, MPI)
// ----------------------------------------------------------------------------
template <class R>
int set_halo_impl(or_ecycle* h, int nloc, const int* local_node, const int* slot, const int* count_ke, int nhalo) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  m.per.on = false;            // a domain of a split mesh runs the phase kernels
  const HPart& P = h->parts[0];
  std::vector<int> hs(m.nnodpad, -1), hn(std::max(nhalo, 1), -1);
  std::vector<unsigned char> ke(m.nnodpad, 1);
  for (int i = 0; i < nloc; ++i) {
    const int n = local_node[i], q = slot[i];
    if (n < 0 || n >= P.numnod || q < 0 || q >= nhalo) return fail(h, OR_E_ARG, "set_halo: node or slot out of range");
    if (hn[q] >= 0) return fail(h, OR_E_ARG, "set_halo: slot given twice");
    const int g = P.node_start + n;
    hs[g] = q;
    hn[q] = g;
    ke[g] = count_ke ? (count_ke[i] ? 1 : 0) : 1;
  }
  dfree(m.halo_slot); dfree(m.halo_node); dfree(m.halo_ke);
  int rc;
  if ((rc = dput(h, m.halo_slot, hs)) || (rc = dput(h, m.halo_node, hn)) || (rc = dput(h, m.halo_ke, ke))) return rc;
  m.nhalo = nhalo;
  return OR_OK;
}

template <class R>
int spmd_begin_impl(or_ecycle* h, or_ecycle_time* t) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  PartTime pt{};
  pt.tt = t->tt; pt.dt2 = t->dt2; pt.dt2old = t->dt2old; pt.dt1 = t->dt1; pt.dt12 = t->dt12;
  pt.ncycle = t->ncycle; pt.ityptst = t->ityptst; pt.neltst = t->neltst;
  PartAcc a0;
  a0.dtkey = ~0ull; a0.dtbits = ~0ull;
  CK(cudaMemcpyAsync(m.time.p, &pt, sizeof(PartTime), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(m.acc.p, &a0, sizeof(PartAcc), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemsetAsync(m.err.p, 0, sizeof(ErrorWord), h->stream));
  CK(cudaStreamSynchronize(h->stream));      // pt and a0 are host locals
  h->spmd_k = 0;
  h->launches = 0;
  return OR_OK;
}

template <class R>
int spmd_elements_impl(or_ecycle* h, void* buf) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const int parity = h->spmd_k & 1;
  int rc = h->tile_hex == 64 ? launch_hex<R, 64>(h, m, parity)
           : h->tile_hex == 128 ? launch_hex<R, 128>(h, m, parity) : launch_hex<R, 256>(h, m, parity);
  if (rc) return rc;
  rc = h->tile_shell == 64 ? launch_shell_npt<R, 64>(h, m, parity)
       : h->tile_shell == 128 ? launch_shell_npt<R, 128>(h, m, parity) : launch_shell_npt<R, 256>(h, m, parity);
  if (rc) return rc;
  halo_pack_kernel<R><<<(unsigned)std::max(1, (m.nhalo + 127) / 128), 128, 0, h->stream>>>(
      m.halo_node.p, m.adsky.p, m.fslot.p, m.mslot.p, m.acc.p + parity, (unsigned char*)buf, m.nhalo);
  CK(cudaGetLastError());
  h->launches++;
  return OR_OK;
}

template <class R>
int spmd_nodes_impl(or_ecycle* h, const void* bufs, int nranks) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const int parity = h->spmd_k & 1;
  NodeArgs<R> a = m.nargs(h);
  a.halo_slot = m.halo_slot.p; a.halo_ke = m.halo_ke.p; a.xbuf = (const unsigned char*)bufs;
  a.xbytes = halo_buffer_bytes<R>(m.nhalo); a.nranks = nranks; a.nhalo = m.nhalo;
  if (node_wide(h, m)) node_kernel_wide<R, NODE_TILE><<<(unsigned)m.ntiles, NODE_TILE, 0, h->stream>>>(a, parity);
  else node_kernel<R, NODE_TILE><<<(unsigned)m.ntiles, NODE_TILE, 0, h->stream>>>(a, parity);
  CK(cudaGetLastError());
  h->launches++;
  h->spmd_k++;
  return OR_OK;
}

template <class R>
int spmd_end_impl(or_ecycle* h, or_ecycle_time* t) {
  Impl<R>& m = *(Impl<R>*)h->impl;
  const int fin = h->spmd_k & 1;
  PartTime pt{};
  ErrorWord ew{};
  const int rc = wait_queued(h);
  if (rc) return rc;
  CK(cudaMemcpyAsync(&pt, m.time.p + fin, sizeof(PartTime), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(&ew, m.err.p, sizeof(ErrorWord), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  t->tt = pt.tt; t->dt1 = pt.dt1; t->dt2 = pt.dt2; t->dt12 = pt.dt12; t->dt2old = pt.dt2old;
  t->ncycle = pt.ncycle; t->ityptst = pt.ityptst; t->neltst = pt.neltst;
  h->next_parity = fin;
  h->spmd_k = -1;
  h->last_code = ew.code;
  h->last_index = ew.index;
  if (ew.code) {
    char b[160];
    snprintf(b, sizeof b, "device error %d at index %d", ew.code, ew.index);
    return fail(h, ew.code, b);
  }
  return OR_OK;
}

int spmd_nhalo(const or_ecycle* h) {
  return h->cfg.precision == OR_PREC_SPLIT ? ((const Impl<float>*)h->impl)->nhalo
                                           : ((const Impl<double>*)h->impl)->nhalo;
}

int spmd_ready(or_ecycle* h, bool running) {
  if (!h) return OR_E_ARG;
  if (!h->finalized) return fail(h, OR_E_STATE, "spmd call before finalize");
  if (spmd_nhalo(h) < 0) return fail(h, OR_E_STATE, "spmd call before set_halo");
  if (running != (h->spmd_k >= 0))
    return fail(h, OR_E_STATE, running ? "spmd cycle outside spmd_begin/end" : "spmd_begin twice");
  cudaSetDevice(h->cfg.device);
  return OR_OK;
}

#define DISPATCH(h, fn, ...) \
  ((h)->cfg.precision == OR_PREC_SPLIT ? fn<float>(h, __VA_ARGS__) : fn<double>(h, __VA_ARGS__))

// ----------------------------------------------------------------------------
// adjoint of the shell cycle (FP64 handles): checkpointed forward sweep, then
// per segment a recompute that stores every cycle's start state, then the
// reverse cycles of the segment from last to first
// ----------------------------------------------------------------------------
struct AdjField {
  void* p;
  size_t bytes, off;
};

struct AdjWork {
  DBuf<AdjGroup> groups; DBuf<int> egroup; DBuf<int4> enodes; DBuf<int> csr_ofs, csr_ent;
  DBuf<double4> lamX, lamD, lamV, lamVR, lamF, lamM, cX, cV, cR;
  DBuf<double> dms, din, lsig, lpla, lthk, lhourg, dA, dthke;
  DBuf<PartTime> tlog;
  DBuf<unsigned char> ckpt, seg, fin;
  std::vector<AdjField> full, slot;
  size_t full_bytes = 0, slot_bytes = 0;
  int ncap = -1, nck_cap = 0, kcap = 0;
  void free_all() {
    dfree(groups); dfree(egroup); dfree(enodes); dfree(csr_ofs); dfree(csr_ent);
    dfree(lamX); dfree(lamD); dfree(lamV); dfree(lamVR); dfree(lamF); dfree(lamM); dfree(cX); dfree(cV); dfree(cR);
    dfree(dms); dfree(din); dfree(lsig); dfree(lpla); dfree(lthk); dfree(lhourg); dfree(dA); dfree(dthke);
    dfree(tlog); dfree(ckpt); dfree(seg); dfree(fin);
  }
};

size_t layout_fields(std::vector<AdjField>& f) {
  size_t off = 0;
  for (auto& x : f) { x.off = off; off += (x.bytes + 255) / 256 * 256; }
  return off;
}

int adj_save(or_ecycle* h, const std::vector<AdjField>& f, unsigned char* buf) {
  for (const auto& x : f)
    if (x.bytes) CK(cudaMemcpyAsync(buf + x.off, x.p, x.bytes, cudaMemcpyDeviceToDevice, h->stream));
  return OR_OK;
}
int adj_restore(or_ecycle* h, const std::vector<AdjField>& f, const unsigned char* buf) {
  for (const auto& x : f)
    if (x.bytes) CK(cudaMemcpyAsync(x.p, buf + x.off, x.bytes, cudaMemcpyDeviceToDevice, h->stream));
  return OR_OK;
}

// device tables and buffers of the adjoint, sized for ncycles / checkpoint
int adj_prepare(or_ecycle* h, Impl<double>& m, int ncycles, int K) {
  if (!h->adj) h->adj = new AdjWork();
  AdjWork& w = *(AdjWork*)h->adj;
  int rc;
  const int nn = m.nnodpad, np = m.sps.nelpad;
  if (!w.groups.p) {
    std::vector<AdjGroup> gr;
    for (auto& g : h->shell) {
      AdjGroup a{};
      orb_adj::ShellParams& P = a.P;
      P.law = g.mat.law; P.npt = g.prop.npt; P.ithk = g.prop.ithk; P.degen = 0;
      P.ishfram = g.prop.ishfram; P.pad = 0;
      P.rho = g.mat.rho0; P.young = g.mat.young; P.nu = g.mat.nu; P.shear = g.mat.shear; P.a11 = g.mat.a11;
      P.a12 = g.mat.a12; P.jc_b = g.mat.jc_b; P.jc_n = g.mat.jc_n; P.sigmax = g.mat.sigmax;
      P.hm = g.prop.hm; P.hf = g.prop.hf; P.hr = g.prop.hr; P.shf = g.prop.shf; P.pressure = g.prop.pressure;
      a.part = g.part; a.has_jca = g.jca.empty() ? 0 : 1; a.jc_a = g.mat.jc_a;
      gr.push_back(a);
    }
    // global corner nodes of each internal element, and the node -> corner CSR
    std::vector<int4> en(np, make_int4(0, 0, 0, 0));
    std::vector<int> cnt(nn + 1, 0);
    for (const PatchInfo& pi : m.sps.info)
      for (int t = 0; t < pi.nel; ++t) {
        const int ie = pi.elem0 + t;
        int g[4];
        for (int k = 0; k < 4; ++k) {
          const int l = m.sps.local[(size_t)ie * 4 + k] & LOCAL_MASK;
          if (l >= pi.nloc) return fail(h, OR_E_STATE, "adjoint: corner outside its patch");
          g[k] = m.sps.nodes[pi.node_ofs + l];
          if (g[k] < 0 || g[k] >= nn) return fail(h, OR_E_STATE, "adjoint: corner node out of range");
          cnt[g[k] + 1]++;
        }
        en[ie] = make_int4(g[0], g[1], g[2], g[3]);
      }
    for (int n = 0; n < nn; ++n) cnt[n + 1] += cnt[n];
    std::vector<int> ent(cnt[nn]), nxt(cnt.begin(), cnt.end() - 1);
    for (int ie = 0; ie < np; ++ie) {
      if (m.sps.elem_group[ie] < 0) continue;
      const int g[4] = {en[ie].x, en[ie].y, en[ie].z, en[ie].w};
      for (int k = 0; k < 4; ++k) ent[nxt[g[k]]++] = 4 * ie + k;
    }
    if ((rc = dput(h, w.groups, gr)) || (rc = dput(h, w.egroup, m.sps.elem_group)) || (rc = dput(h, w.enodes, en)) ||
        (rc = dput(h, w.csr_ofs, cnt)) || (rc = dput(h, w.csr_ent, ent)))
      return rc;
    const size_t n4 = (size_t)nn, c4 = 4 * (size_t)np;
    if ((rc = dalloc(h, w.lamX, n4)) || (rc = dalloc(h, w.lamD, n4)) || (rc = dalloc(h, w.lamV, n4)) ||
        (rc = dalloc(h, w.lamVR, n4)) || (rc = dalloc(h, w.lamF, n4)) || (rc = dalloc(h, w.lamM, n4)) ||
        (rc = dalloc(h, w.cX, c4)) || (rc = dalloc(h, w.cV, c4)) || (rc = dalloc(h, w.cR, c4)) ||
        (rc = dalloc(h, w.dms, n4)) || (rc = dalloc(h, w.din, n4)) || (rc = dalloc(h, w.lsig, m.ssig.n)) ||
        (rc = dalloc(h, w.lpla, m.spla.n)) || (rc = dalloc(h, w.lthk, (size_t)np)) ||
        (rc = dalloc(h, w.lhourg, 3 * (size_t)np)) || (rc = dalloc(h, w.dA, (size_t)np)) ||
        (rc = dalloc(h, w.dthke, (size_t)np)))
      return rc;
    // the full state (checkpoints, end state) and the per-cycle slot state
    w.full = {{m.X.p, m.X.n * sizeof(double4), 0}, {m.DX.p, m.DX.n * sizeof(double), 0},
              {m.DY.p, m.DY.n * sizeof(double), 0}, {m.DZ.p, m.DZ.n * sizeof(double), 0},
              {m.V.p, m.V.n * sizeof(double4), 0}, {m.VR.p, m.VR.n * sizeof(double4), 0},
              {m.ssig.p, m.ssig.n * sizeof(double), 0}, {m.spla.p, m.spla.n * sizeof(double), 0},
              {m.sthk.p, m.sthk.n * sizeof(double), 0}, {m.shourg.p, m.shourg.n * sizeof(double), 0},
              {m.seint.p, m.seint.n * sizeof(double), 0}, {m.sehour.p, m.sehour.n * sizeof(double), 0},
              {m.swpla.p, m.swpla.n * sizeof(double), 0}, {m.ekin.p, m.ekin.n * sizeof(double), 0},
              {m.ekinr.p, m.ekinr.n * sizeof(double), 0}};
    w.slot = {{m.X.p, m.X.n * sizeof(double4), 0}, {m.V.p, m.V.n * sizeof(double4), 0},
              {m.VR.p, m.VR.n * sizeof(double4), 0}, {m.ssig.p, m.ssig.n * sizeof(double), 0},
              {m.spla.p, m.spla.n * sizeof(double), 0}, {m.sthk.p, m.sthk.n * sizeof(double), 0},
              {m.shourg.p, m.shourg.n * sizeof(double), 0}};
    w.full_bytes = layout_fields(w.full);
    w.slot_bytes = layout_fields(w.slot);
    if ((rc = dalloc(h, w.fin, w.full_bytes))) return rc;
  }
  const int nck = (ncycles + K - 1) / K;
  if (ncycles > w.ncap) {
    dfree(w.tlog);
    if ((rc = dalloc(h, w.tlog, (size_t)(ncycles + 1) * m.nparts))) return rc;
    w.ncap = ncycles;
  }
  if (nck > w.nck_cap) {
    dfree(w.ckpt);
    if ((rc = dalloc(h, w.ckpt, (size_t)nck * w.full_bytes))) return rc;
    w.nck_cap = nck;
  }
  if (K > w.kcap) {
    dfree(w.seg);
    if ((rc = dalloc(h, w.seg, (size_t)(K + 1) * w.slot_bytes))) return rc;
    w.kcap = K;
  }
  return OR_OK;
}

int adj_check_error(or_ecycle* h, Impl<double>& m) {
  ErrorWord ew{};
  const int rc = wait_queued(h);
  if (rc) return rc;
  CK(cudaMemcpyAsync(&ew, m.err.p, sizeof(ErrorWord), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->last_code = ew.code;
  h->last_index = ew.index;
  if (ew.code) {
    char buf[160];
    snprintf(buf, sizeof buf, "device error %d at index %d", ew.code, ew.index);
    return fail(h, ew.code, buf);
  }
  return OR_OK;
}

double adj_plastic_work(or_ecycle* h) {
  double s = 0.0;
  for (int p = 0; p < (int)h->parts.size(); ++p) {
    or_energies e{};
    if (energies_impl<double>(h, p, &e) == OR_OK) s += e.plastic_work;
  }
  return s;
}

template <int NP>
int launch_adj_shell(or_ecycle* h, const AdjShellArgs& a) {
  adj_shell_kernel<NP><<<(unsigned)((a.nelpad + ADJ_SHELL_THREADS - 1) / ADJ_SHELL_THREADS), ADJ_SHELL_THREADS, 0,
                         h->stream>>>(a);
  CK(cudaGetLastError());
  h->launches++;
  return OR_OK;
}

int adjoint_impl(or_ecycle* h, int N, const or_adjoint_response* r, or_ecycle_time* t, double* J, double* dJ_dA,
                 double* dJ_dthk, double* dJ_dms, double* dJ_din) {
  Impl<double>& m = *(Impl<double>*)h->impl;
  const int K = r->checkpoint > 0 ? r->checkpoint : 50;
  int rc = adj_prepare(h, m, N, K);
  if (rc) return rc;
  AdjWork& w = *(AdjWork*)h->adj;
  const int np = m.nparts, nn = m.nnodpad, nelpad = m.sps.nelpad;
  int gnode = -1;
  if (r->node >= 0) gnode = h->parts[r->part].node_start + r->node;
  // ---- forward sweep with checkpoints ----
  std::vector<PartTime> pt(np);
  for (int p = 0; p < np; ++p) {
    pt[p].tt = t[p].tt; pt[p].dt2 = t[p].dt2; pt[p].dt2old = t[p].dt2old; pt[p].dt1 = t[p].dt1;
    pt[p].dt12 = t[p].dt12; pt[p].ncycle = t[p].ncycle; pt[p].ityptst = t[p].ityptst; pt[p].neltst = t[p].neltst;
    pt[p].pad = 0;
  }
  const double wp0 = adj_plastic_work(h);
  h->launches = 0;
  CK(cudaMemcpyAsync(m.time.p, pt.data(), np * sizeof(PartTime), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(w.tlog.p, pt.data(), np * sizeof(PartTime), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemsetAsync(m.acc.p, 0xff, np * sizeof(PartAcc), h->stream));
  CK(cudaMemsetAsync(m.err.p, 0, sizeof(ErrorWord), h->stream));
  for (int c = 0; c < N; ++c) {
    if (c % K == 0 && (rc = adj_save(h, w.full, w.ckpt.p + (size_t)(c / K) * w.full_bytes))) return rc;
    if ((rc = launch_cycle<double>(h, m, c & 1, nullptr))) return rc;
    CK(cudaMemcpyAsync(w.tlog.p + (size_t)(c + 1) * np, m.time.p + ((c + 1) & 1) * np, np * sizeof(PartTime),
                       cudaMemcpyDeviceToDevice, h->stream));
  }
  if ((rc = adj_save(h, w.full, w.fin.p))) return rc;
  if ((rc = adj_check_error(h, m))) return rc;
  const double wp1 = adj_plastic_work(h);
  double dval = 0.0;
  if (gnode >= 0) {
    const double* D = r->comp == 0 ? m.DX.p : r->comp == 1 ? m.DY.p : m.DZ.p;
    CK(cudaMemcpy(&dval, D + gnode, sizeof(double), cudaMemcpyDeviceToHost));
  }
  const double Jval = r->w_disp * dval + r->w_plastic * (wp1 - wp0);
  // ---- adjoint state at the end ----
  CK(cudaMemsetAsync(w.lamX.p, 0, nn * sizeof(double4), h->stream));
  CK(cudaMemsetAsync(w.lamD.p, 0, nn * sizeof(double4), h->stream));
  CK(cudaMemsetAsync(w.lamV.p, 0, nn * sizeof(double4), h->stream));
  CK(cudaMemsetAsync(w.lamVR.p, 0, nn * sizeof(double4), h->stream));
  CK(cudaMemsetAsync(w.dms.p, 0, nn * sizeof(double), h->stream));
  CK(cudaMemsetAsync(w.din.p, 0, nn * sizeof(double), h->stream));
  CK(cudaMemsetAsync(w.lsig.p, 0, w.lsig.n * sizeof(double), h->stream));
  CK(cudaMemsetAsync(w.lpla.p, 0, w.lpla.n * sizeof(double), h->stream));
  CK(cudaMemsetAsync(w.lthk.p, 0, w.lthk.n * sizeof(double), h->stream));
  CK(cudaMemsetAsync(w.lhourg.p, 0, w.lhourg.n * sizeof(double), h->stream));
  CK(cudaMemsetAsync(w.dA.p, 0, w.dA.n * sizeof(double), h->stream));
  CK(cudaMemsetAsync(w.dthke.p, 0, w.dthke.n * sizeof(double), h->stream));
  if (gnode >= 0) {
    const double wd = r->w_disp;
    CK(cudaMemcpyAsync((double*)(w.lamD.p + gnode) + r->comp, &wd, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));      // wd is a host local
  }
  // ---- reverse, segment by segment ----
  const int nseg = (N + K - 1) / K;
  const unsigned nb_node = (unsigned)((nn + 127) / 128);
  const AdjField& fX = w.slot[0];
  const AdjField& fV = w.slot[1];
  const AdjField& fVR = w.slot[2];
  const AdjField& fS = w.slot[3];
  const AdjField& fP = w.slot[4];
  const AdjField& fT = w.slot[5];
  const AdjField& fH = w.slot[6];
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int c0 = sg * K, c1 = std::min(N, c0 + K);
    if ((rc = adj_restore(h, w.full, w.ckpt.p + (size_t)sg * w.full_bytes))) return rc;
    CK(cudaMemcpyAsync(m.time.p + (c0 & 1) * np, w.tlog.p + (size_t)c0 * np, np * sizeof(PartTime),
                       cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemsetAsync(m.acc.p + (c0 & 1) * np, 0xff, np * sizeof(PartAcc), h->stream));
    for (int c = c0; c < c1; ++c) {
      if ((rc = adj_save(h, w.slot, w.seg.p + (size_t)(c - c0) * w.slot_bytes))) return rc;
      if ((rc = launch_cycle<double>(h, m, c & 1, nullptr))) return rc;
    }
    if ((rc = adj_save(h, w.slot, w.seg.p + (size_t)(c1 - c0) * w.slot_bytes))) return rc;
    for (int c = c1 - 1; c >= c0; --c) {
      unsigned char* s0 = w.seg.p + (size_t)(c - c0) * w.slot_bytes;
      unsigned char* s1 = s0 + w.slot_bytes;
      AdjNodeArgs na;
      na.parts = m.partd.p; na.tile_part = m.tile_part.p; na.code = m.code.p;
      na.Xn = (const double4*)(s0 + fX.off); na.Vn = (const double4*)(s0 + fV.off);
      na.Vn1 = (const double4*)(s1 + fV.off); na.VRn = (const double4*)(s0 + fVR.off);
      na.VRn1 = (const double4*)(s1 + fVR.off); na.tnext = w.tlog.p + (size_t)(c + 1) * np;
      na.lamX = w.lamX.p; na.lamD = w.lamD.p; na.lamV = w.lamV.p; na.lamVR = w.lamVR.p;
      na.lamF = w.lamF.p; na.lamM = w.lamM.p; na.dms = w.dms.p; na.din = w.din.p;
      na.nnodpad = nn; na.node_tile = NODE_TILE;
      na.skew_of = m.skew_of.p; na.skews = m.skw.p;
      adj_node_pre_kernel<<<nb_node, 128, 0, h->stream>>>(na);
      CK(cudaGetLastError());
      AdjShellArgs sa;
      sa.groups = w.groups.p; sa.egroup = w.egroup.p; sa.enodes = w.enodes.p; sa.degen = m.sdegen.p;
      sa.Xn = na.Xn; sa.Vn = na.Vn; sa.VRn = na.VRn;
      sa.sig = (const double*)(s0 + fS.off); sa.pla = (const double*)(s0 + fP.off);
      sa.thk = (const double*)(s0 + fT.off); sa.thke = m.sthke.p; sa.hourg = (const double*)(s0 + fH.off);
      sa.jca = m.sjca.p; sa.tcur = w.tlog.p + (size_t)c * np; sa.lamF = w.lamF.p; sa.lamM = w.lamM.p;
      sa.lsig = w.lsig.p; sa.lpla = w.lpla.p; sa.lthk = w.lthk.p; sa.lhourg = w.lhourg.p; sa.dA = w.dA.p;
      sa.dthke = w.dthke.p; sa.cX = w.cX.p; sa.cV = w.cV.p; sa.cR = w.cR.p; sa.zw = m.zw.p;
      sa.w_plastic = r->w_plastic; sa.nelpad = nelpad;
      rc = m.uniform_npt == 5 ? launch_adj_shell<5>(h, sa) : launch_adj_shell<10>(h, sa);
      if (rc) return rc;
      AdjPostArgs pa;
      pa.ofs = w.csr_ofs.p; pa.ent = w.csr_ent.p; pa.cX = w.cX.p; pa.cV = w.cV.p; pa.cR = w.cR.p;
      pa.lamX = w.lamX.p; pa.lamV = w.lamV.p; pa.lamVR = w.lamVR.p; pa.nnodpad = nn;
      adj_node_post_kernel<<<nb_node, 128, 0, h->stream>>>(pa);
      CK(cudaGetLastError());
      h->launches += 3;
    }
  }
  // ---- back to the end state of the forward sweep ----
  if ((rc = adj_restore(h, w.full, w.fin.p))) return rc;
  CK(cudaMemcpyAsync(m.time.p + (N & 1) * np, w.tlog.p + (size_t)N * np, np * sizeof(PartTime),
                     cudaMemcpyDeviceToDevice, h->stream));
  if ((rc = adj_check_error(h, m))) return rc;
  // ---- outputs in user order ----
  std::vector<PartTime> tend(np);
  CK(cudaMemcpy(tend.data(), w.tlog.p + (size_t)N * np, np * sizeof(PartTime), cudaMemcpyDeviceToHost));
  if (dJ_dA || dJ_dthk) {
    auto dA = d2h(w.dA.p, (size_t)nelpad);
    auto dte = d2h(w.dthke.p, (size_t)nelpad);
    auto lth = d2h(w.lthk.p, (size_t)nelpad);
    size_t o = 0;
    for (auto& g : h->shell) {
      for (int ue = 0; ue < g.nel; ++ue) {
        const int ie = g.internal[ue];
        if (dJ_dA) dJ_dA[o + ue] = g.mat.law == OR_LAW_JOHNSON_COOK ? dA[ie] : 0.0;
        if (dJ_dthk) dJ_dthk[o + ue] = lth[ie] + dte[ie];
      }
      o += g.nel;
    }
  }
  if (dJ_dms || dJ_din) {
    auto dm = d2h(w.dms.p, (size_t)nn);
    auto di = d2h(w.din.p, (size_t)nn);
    size_t o = 0;
    for (auto& P : h->parts) {
      for (int i = 0; i < P.numnod; ++i) {
        if (dJ_dms) dJ_dms[o + i] = dm[P.node_start + i];
        if (dJ_din) dJ_din[o + i] = di[P.node_start + i];
      }
      o += P.numnod;
    }
  }
  CK(cudaGetLastError());
  for (int p = 0; p < np; ++p) {
    t[p].tt = tend[p].tt; t[p].dt1 = tend[p].dt1; t[p].dt2 = tend[p].dt2; t[p].dt12 = tend[p].dt12;
    t[p].dt2old = tend[p].dt2old; t[p].ncycle = tend[p].ncycle; t[p].ityptst = tend[p].ityptst;
    t[p].neltst = tend[p].neltst;
  }
  if (J) *J = Jval;
  return OR_OK;
}

void adj_destroy(or_ecycle* h) {
  if (!h->adj) return;
  AdjWork* w = (AdjWork*)h->adj;
  w->free_all();
  delete w;
  h->adj = nullptr;
}

bool bad_ptr(const void* p) { return p == nullptr; }

}  // namespace

extern "C" {

int or_ecycle_create(const or_ecycle_config* cfg, or_ecycle** out) {
  if (!cfg || !out) return OR_E_ARG;
  if (cfg->precision != OR_PREC_FP64 && cfg->precision != OR_PREC_SPLIT) return OR_E_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return OR_E_CUDA;
  if (cfg->device < 0 || cfg->device >= ndev) return OR_E_ARG;
  or_ecycle* h = new or_ecycle();
  h->cfg = *cfg;
  if (h->cfg.dt_growth <= 0) h->cfg.dt_growth = (double)1.1f;
  if (h->cfg.dtmx <= 0) h->cfg.dtmx = 1e20;
  auto tile_ok = [](int b) { return b == 64 || b == 128 || b == 256; };
  if (tile_ok(h->cfg.block_hex)) h->tile_hex = h->cfg.block_hex;
  if (tile_ok(h->cfg.block_shell)) h->tile_shell = h->cfg.block_shell;
  if (const char* s = std::getenv("OR_ECYCLE_PDL")) h->pdl = std::atoi(s) != 0;
  if (const char* s = std::getenv("OR_ECYCLE_SHELL_STAGED")) h->shell_staged = std::atoi(s) != 0 ? 1 : 0;
  if (cudaSetDevice(cfg->device) != cudaSuccess || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return OR_E_CUDA;
  }
  cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, cfg->device);
  *out = h;
  return OR_OK;
}

int or_ecycle_destroy(or_ecycle* h) {
  if (!h) return OR_E_ARG;
  cudaSetDevice(h->cfg.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  adj_destroy(h);
  if (h->cfg.precision == OR_PREC_SPLIT) destroy_impl<float>(h); else destroy_impl<double>(h);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return OR_OK;
}

const char* or_ecycle_last_error(const or_ecycle* h) { return h ? h->err.c_str() : "null handle"; }

int or_ecycle_add_part(or_ecycle* h, int numnod, const double* x, const double* v, const double* vr, const double* ms,
                       const double* in, const int* icodt, const int* icodr, int* part) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "add_part after finalize");
  if (numnod <= 0 || bad_ptr(x) || bad_ptr(v) || bad_ptr(ms) || bad_ptr(icodt) || bad_ptr(part))
    return fail(h, OR_E_ARG, "add_part: null array or empty part");
  HPart P;
  P.numnod = numnod;
  P.x.assign(x, x + 3 * (size_t)numnod);
  P.v.assign(v, v + 3 * (size_t)numnod);
  P.vr.assign(3 * (size_t)numnod, 0.0);
  if (vr) P.vr.assign(vr, vr + 3 * (size_t)numnod);
  P.ms.assign(ms, ms + numnod);
  P.in.assign(numnod, 0.0);
  if (in) P.in.assign(in, in + numnod);
  P.icodt.assign(icodt, icodt + numnod);
  P.icodr.assign(numnod, 0);
  if (icodr) P.icodr.assign(icodr, icodr + numnod);
  for (int i = 0; i < 3 * numnod; ++i)
    if (!std::isfinite(P.x[i]) || !std::isfinite(P.v[i])) return fail(h, OR_E_ARG, "add_part: non-finite X or V");
  h->parts.push_back(std::move(P));
  *part = (int)h->parts.size() - 1;
  return OR_OK;
}

int or_ecycle_add_hex_group(or_ecycle* h, int part, int nel, const int* ixs, const or_material* mat,
                            const or_solid_prop* prop, const double* vol0, int* group) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "add_hex_group after finalize");
  if (part < 0 || part >= (int)h->parts.size() || nel <= 0 || !ixs || !mat || !prop || !group)
    return fail(h, OR_E_ARG, "add_hex_group: bad argument");
  if (mat->law != OR_LAW_ELASTIC && mat->law != OR_LAW_JOHNSON_COOK) return fail(h, OR_E_UNSUPPORTED, "hex law");
  if (prop->jcvt != 0 && prop->jcvt != 1) return fail(h, OR_E_UNSUPPORTED, "hex frame other than global or convected");
  HHex g;
  g.part = part; g.nel = nel; g.mat = *mat; g.prop = *prop;
  HPart& P = h->parts[part];
  g.gofs = P.nel_solid;
  g.conn.resize(8 * (size_t)nel);
  for (int e = 0; e < nel; ++e)
    for (int k = 0; k < 8; ++k) {
      const int n = ixs[11 * (size_t)e + 1 + k] - 1;   // IXS rows 2..9, Fortran numbering
      if (n < 0 || n >= P.numnod) return fail(h, OR_E_ARG, "add_hex_group: node index out of range in IXS");
      g.conn[8 * (size_t)e + k] = n;
    }
  g.vol0.resize(nel);
  for (int e = 0; e < nel; ++e) {
    double v;
    if (vol0) v = vol0[e];
    else {
      const int* c = &g.conn[8 * (size_t)e];
      auto X = [&](int k, int q) { return P.x[3 * (size_t)c[k] + q]; };
      double d[4][3];
      const int pr[4][2] = {{6, 0}, {7, 1}, {4, 2}, {5, 3}};
      for (int a = 0; a < 4; ++a) for (int q = 0; q < 3; ++q) d[a][q] = X(pr[a][0], q) - X(pr[a][1], q);
      double j1[3], j4[3], j7[3];
      for (int q = 0; q < 3; ++q) {
        j1[q] = d[0][q] + d[1][q] - d[2][q] - d[3][q];
        j4[q] = d[0][q] + d[3][q] + d[1][q] + d[2][q];
        j7[q] = d[0][q] + d[3][q] - d[1][q] - d[2][q];
      }
      v = (j1[0] * (j4[1] * j7[2] - j4[2] * j7[1]) + j1[1] * (j4[2] * j7[0] - j4[0] * j7[2]) +
           j1[2] * (j4[0] * j7[1] - j4[1] * j7[0])) / 64.0;
    }
    if (!(v > 0)) return fail(h, OR_E_NEGVOL, "add_hex_group: non-positive initial volume");
    g.vol0[e] = v;
  }
  P.nel_solid += nel;
  h->hex.push_back(std::move(g));
  *group = (int)h->hex.size() - 1;
  return OR_OK;
}

int or_ecycle_add_shell_group(or_ecycle* h, int part, int nel, const int* ixc, const or_material* mat,
                              const or_shell_prop* prop, const double* thke, int* group) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "add_shell_group after finalize");
  if (part < 0 || part >= (int)h->parts.size() || nel <= 0 || !ixc || !mat || !prop || !group)
    return fail(h, OR_E_ARG, "add_shell_group: bad argument");
  if (prop->npt < 1 || prop->npt > 10) return fail(h, OR_E_UNSUPPORTED, "shell npt outside 1..10");
  if (prop->ipla < 0 || prop->ipla > 2) return fail(h, OR_E_UNSUPPORTED, "shell IPLA outside 0..2");
  if (prop->ishfram != 0 && prop->ishfram != 2) return fail(h, OR_E_UNSUPPORTED, "shell ISHFRAM other than 0 or 2");
  if (prop->ishell < 0 || prop->ishell > 4) return fail(h, OR_E_UNSUPPORTED, "shell Ishell outside 1..4");
  if (!(prop->dn >= 0)) return fail(h, OR_E_ARG, "shell Dn negative");
  if (mat->law != OR_LAW_ELASTIC && mat->law != OR_LAW_JOHNSON_COOK) return fail(h, OR_E_UNSUPPORTED, "shell law");
  HShell g;
  g.part = part; g.nel = nel; g.mat = *mat; g.prop = *prop;
  HPart& P = h->parts[part];
  g.gofs = P.nel_shell;
  g.conn.resize(4 * (size_t)nel);
  for (int e = 0; e < nel; ++e)
    for (int k = 0; k < 4; ++k) {
      const int n = ixc[7 * (size_t)e + 1 + k] - 1;   // IXC rows 2..5
      if (n < 0 || n >= P.numnod) return fail(h, OR_E_ARG, "add_shell_group: node index out of range in IXC");
      g.conn[4 * (size_t)e + k] = n;
    }
  g.thke.resize(nel);
  for (int e = 0; e < nel; ++e) {
    g.thke[e] = thke ? thke[e] : prop->thk;
    if (!(g.thke[e] > 0)) return fail(h, OR_E_ARG, "add_shell_group: non-positive thickness");
  }
  P.nel_shell += nel;
  P.has_rot = true;
  h->shell.push_back(std::move(g));
  *group = (int)h->shell.size() - 1;
  return OR_OK;
}

int or_ecycle_set_shell_yield(or_ecycle* h, int group, const double* jc_a) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "set_shell_yield after finalize");
  if (group < 0 || group >= (int)h->shell.size() || !jc_a) return fail(h, OR_E_ARG, "set_shell_yield: bad argument");
  HShell& g = h->shell[group];
  g.jca.assign(jc_a, jc_a + g.nel);
  return OR_OK;
}

int or_ecycle_add_rlink(or_ecycle* h, int part, int nnod, const int* nodes, int ic, int icr, int* link) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "add_rlink after finalize");
  if (part < 0 || part >= (int)h->parts.size() || nnod < 1 || !nodes || ic < 0 || ic > 7 || icr < 0 || icr > 7)
    return fail(h, OR_E_ARG, "add_rlink: bad argument");
  HLink L;
  L.part = part; L.ic = ic; L.icr = icr;
  std::vector<char> seen(h->parts[part].numnod, 0);
  for (auto& o : h->links)
    if (o.part == part) for (int n : o.nodes) seen[n] = 1;
  for (int i = 0; i < nnod; ++i) {
    const int n = nodes[i] - 1;
    if (n < 0 || n >= h->parts[part].numnod) return fail(h, OR_E_ARG, "add_rlink: node number out of range");
    if (seen[n]) return fail(h, OR_E_UNSUPPORTED, "add_rlink: node already in a rigid link");
    seen[n] = 1;
    L.nodes.push_back(n);
  }
  if (icr && !h->parts[part].has_rot) return fail(h, OR_E_ARG, "add_rlink: rotations on a part without them");
  h->links.push_back(std::move(L));
  if (link) *link = (int)h->links.size() - 1;
  return OR_OK;
}

int or_ecycle_add_rbody(or_ecycle* h, int part, int master, int nsl, const int* slaves, const double* rby12,
                        int* body) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "add_rbody after finalize");
  if (part < 0 || part >= (int)h->parts.size() || !slaves || !rby12 || nsl < 3)
    return fail(h, OR_E_ARG, "add_rbody: bad argument (at least three secondary nodes)");
  HPart& P = h->parts[part];
  std::vector<char> seen(P.numnod, 0);
  for (auto& o : h->rbodies)
    if (o.part == part) {
      seen[o.master] = 1;
      for (int n : o.slaves) seen[n] = 1;
    }
  HRBody B;
  B.part = part;
  B.master = master - 1;
  if (B.master < 0 || B.master >= P.numnod) return fail(h, OR_E_ARG, "add_rbody: main node out of range");
  if (seen[B.master]) return fail(h, OR_E_UNSUPPORTED, "add_rbody: node already in a rigid body");
  seen[B.master] = 1;
  if (P.icodr[B.master] != 0) return fail(h, OR_E_UNSUPPORTED, "add_rbody: rotational BCS on the main node");
  for (int i = 0; i < nsl; ++i) {
    const int n = slaves[i] - 1;
    if (n < 0 || n >= P.numnod) return fail(h, OR_E_ARG, "add_rbody: secondary node out of range");
    if (seen[n]) return fail(h, OR_E_UNSUPPORTED, "add_rbody: node already in a rigid body");
    seen[n] = 1;
    B.slaves.push_back(n);
  }
  for (int k = 0; k < 12; ++k) B.rby[k] = rby12[k];
  if (!(rby12[9] > 0 && rby12[10] > 0 && rby12[11] > 0)) return fail(h, OR_E_ARG, "add_rbody: principal inertias");
  P.has_rot = true;                  // the main node's rotation (VR, IN)
  h->rbodies.push_back(std::move(B));
  if (body) *body = (int)h->rbodies.size() - 1;
  return OR_OK;
}

int or_ecycle_set_rlink(or_ecycle* h, int link, int ic, int icr) {
  if (!h) return OR_E_ARG;
  if (link < 0 || link >= (int)h->links.size() || ic < 0 || ic > 7 || icr < 0 || icr > 7)
    return fail(h, OR_E_ARG, "set_rlink: bad argument");
  HLink& L = h->links[link];
  if (icr && !h->parts[L.part].has_rot) return fail(h, OR_E_ARG, "set_rlink: rotations on a part without them");
  L.ic = ic; L.icr = icr;
  if (!h->finalized) return OR_OK;
  cudaSetDevice(h->cfg.device);
  int first = 0;
  for (int l = 0; l < link; ++l) first += (int)h->links[l].nodes.size();
  LinkDesc d;
  d.first = first; d.count = (int)L.nodes.size(); d.ic = ic; d.icr = icr;
  LinkDesc* dst = h->cfg.precision == OR_PREC_SPLIT ? ((Impl<float>*)h->impl)->linkd.p : ((Impl<double>*)h->impl)->linkd.p;
  CK(cudaMemcpyAsync(dst + link, &d, sizeof(LinkDesc), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return OR_OK;
}

int or_ecycle_add_function(or_ecycle* h, int npts, const double* x, const double* y, int* func) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "add_function after finalize");
  if (npts < 1 || !x || !y) return fail(h, OR_E_ARG, "add_function: bad argument");
  for (int i = 1; i < npts; ++i)
    if (!(x[i] > x[i - 1])) return fail(h, OR_E_ARG, "add_function: abscissae not strictly ascending");
  h->fx.emplace_back(x, x + npts);
  h->fy.emplace_back(y, y + npts);
  if (func) *func = (int)h->fx.size() - 1;
  return OR_OK;
}

int or_ecycle_add_skew(or_ecycle* h, const double* axes9, int* skew) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "add_skew after finalize");
  if (!axes9) return fail(h, OR_E_ARG, "add_skew: bad argument");
  std::array<double, 9> a;
  for (int k = 0; k < 9; ++k) a[k] = axes9[k];
  h->skews.push_back(a);
  if (skew) *skew = (int)h->skews.size() - 1;
  return OR_OK;
}

int or_ecycle_add_cload(or_ecycle* h, int part, int nnod, const int* nodes, int dir, int skew, int func,
                        double ascale_x, double fscale, int* load) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "add_cload after finalize");
  if (part < 0 || part >= (int)h->parts.size() || nnod < 1 || !nodes || dir < 1 || dir > 6 || func < 0 ||
      func >= (int)h->fx.size() || skew < -1 || skew >= (int)h->skews.size() || ascale_x == 0.0)
    return fail(h, OR_E_ARG, "add_cload: bad argument");
  HPart& P = h->parts[part];
  if (dir > 3 && !P.has_rot) return fail(h, OR_E_ARG, "add_cload: moment on a part without rotations");
  if (load) *load = (int)h->loads.size();
  for (int i = 0; i < nnod; ++i) {
    if (nodes[i] < 1 || nodes[i] > P.numnod) return fail(h, OR_E_ARG, "add_cload: node number out of range");
    HLoad L;
    L.type = 0; L.part = part; L.func = func; L.dir = dir; L.skew = skew; L.node[0] = nodes[i] - 1;
    L.fcx = 1.0 / ascale_x; L.fcy = fscale;
    h->loads.push_back(L);
  }
  return OR_OK;
}

int or_ecycle_add_pload(or_ecycle* h, int part, int nseg, const int* seg, int func, double ascale_x, double fscale,
                        int* load) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "add_pload after finalize");
  if (part < 0 || part >= (int)h->parts.size() || nseg < 1 || !seg || func < 0 || func >= (int)h->fx.size() ||
      ascale_x == 0.0)
    return fail(h, OR_E_ARG, "add_pload: bad argument");
  const HPart& P = h->parts[part];
  if (load) *load = (int)h->loads.size();
  for (int i = 0; i < nseg; ++i) {
    HLoad L;
    L.type = 1; L.part = part; L.func = func; L.fcx = 1.0 / ascale_x; L.fcy = fscale;
    for (int k = 0; k < 4; ++k) {
      const int n = seg[4 * i + k];
      if (k == 3 && n == 0) break;          // triangle
      if (n < 1 || n > P.numnod) return fail(h, OR_E_ARG, "add_pload: node number out of range");
      L.node[k] = n - 1;
    }
    h->loads.push_back(L);
  }
  return OR_OK;
}

int or_ecycle_set_bcs_skew(or_ecycle* h, int part, const int* skew) {
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "set_bcs_skew after finalize");
  if (part < 0 || part >= (int)h->parts.size() || !skew) return fail(h, OR_E_ARG, "set_bcs_skew: bad argument");
  HPart& P = h->parts[part];
  for (int i = 0; i < P.numnod; ++i)
    if (skew[i] < -1 || skew[i] >= (int)h->skews.size()) return fail(h, OR_E_ARG, "set_bcs_skew: skew out of range");
  P.iskew.assign(skew, skew + P.numnod);
  return OR_OK;
}

int or_ecycle_finalize(or_ecycle* h) {
  Trace tr("or_ecycle_finalize");
  if (!h) return OR_E_ARG;
  if (h->finalized) return fail(h, OR_E_STATE, "finalize called twice");
  if (h->parts.empty()) return fail(h, OR_E_STATE, "finalize without parts");
  if (cudaSetDevice(h->cfg.device) != cudaSuccess) return fail(h, OR_E_CUDA, "cudaSetDevice");
  int rc = h->cfg.precision == OR_PREC_SPLIT ? finalize_impl<float>(h) : finalize_impl<double>(h);
  if (rc) return rc;
  h->finalized = true;
  return OR_OK;
}

int or_ecycle_reset(or_ecycle* h) {
  Trace tr("or_ecycle_reset");
  if (!h) return OR_E_ARG;
  if (!h->finalized) return fail(h, OR_E_STATE, "reset before finalize");
  cudaSetDevice(h->cfg.device);
  h->next_parity = 0;
  for (auto& P : h->parts) P.ehour0 = P.wpla0 = P.wext0 = 0.0;
  return h->cfg.precision == OR_PREC_SPLIT ? reset_impl<float>(h) : reset_impl<double>(h);
}

int or_ecycle_step(or_ecycle* h, int ncycles, or_ecycle_time* t) {
  Trace tr("or_ecycle_step");
  if (!h) return OR_E_ARG;
  if (!h->finalized) return fail(h, OR_E_STATE, "step before finalize");
  if (ncycles < 0 || !t) return fail(h, OR_E_ARG, "step: bad argument");
  if (ncycles == 0) return OR_OK;
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, step_impl, ncycles, t);
}

int or_ecycle_adjoint(or_ecycle* h, int ncycles, const or_adjoint_response* r, or_ecycle_time* t, double* J,
                      double* dJ_dA, double* dJ_dthk, double* dJ_dms, double* dJ_din) {
  Trace tr("or_ecycle_adjoint");
  if (!h) return OR_E_ARG;
  if (!h->finalized) return fail(h, OR_E_STATE, "adjoint before finalize");
  if (ncycles <= 0 || !r || !t) return fail(h, OR_E_ARG, "adjoint: bad argument");
  if (h->cfg.precision != OR_PREC_FP64) return fail(h, OR_E_UNSUPPORTED, "adjoint: FP64 handles only");
  if (!h->hex.empty() || h->shell.empty()) return fail(h, OR_E_UNSUPPORTED, "adjoint: shell groups only");
  if (!h->links.empty()) return fail(h, OR_E_UNSUPPORTED, "adjoint: rigid links");
  if (!h->rbodies.empty()) return fail(h, OR_E_UNSUPPORTED, "adjoint: rigid bodies");
  for (const HShell& g : h->shell) {
    if (g.prop.ipla != 0) return fail(h, OR_E_UNSUPPORTED, "adjoint: IPLA 1 and 2 (the reverse follows the radial return)");
    if (shell_ihbe(g.prop.ishell, g.prop.npt) != 1 || g.prop.npt == 1)
      return fail(h, OR_E_UNSUPPORTED, "adjoint: Ishell 1 with 2 to 10 points only (the reverse follows CHVIS3)");
  }
  for (auto& L : h->loads)     // /CLOAD forces depend on time only: no reverse terms
    if (L.type != 0) return fail(h, OR_E_UNSUPPORTED, "adjoint: /PLOAD follower loads");

  if (r->node >= 0) {
    if (r->part < 0 || r->part >= (int)h->parts.size() || r->node >= h->parts[r->part].numnod || r->comp < 0 ||
        r->comp > 2)
      return fail(h, OR_E_ARG, "adjoint: response node out of range");
  }
  cudaSetDevice(h->cfg.device);
  return adjoint_impl(h, ncycles, r, t, J, dJ_dA, dJ_dthk, dJ_dms, dJ_din);
}

int or_ecycle_set_halo(or_ecycle* h, int part, int nloc, const int* local_node, const int* halo_slot,
                       const int* count_ke, int nhalo) {
  if (!h) return OR_E_ARG;
  if (!h->finalized) return fail(h, OR_E_STATE, "set_halo before finalize");
  if (h->parts.size() != 1 || part != 0) return fail(h, OR_E_UNSUPPORTED, "set_halo: one part per handle");
  if (!h->links.empty()) return fail(h, OR_E_UNSUPPORTED, "set_halo: rigid links across domains");
  if (!h->rbodies.empty()) return fail(h, OR_E_UNSUPPORTED, "set_halo: rigid bodies across domains");
  if (!h->loads.empty()) return fail(h, OR_E_UNSUPPORTED, "set_halo: /CLOAD or /PLOAD loads");
  if (h->spmd_k >= 0) return fail(h, OR_E_STATE, "set_halo inside spmd_begin/end");
  if (nloc < 0 || nhalo < 0 || nloc > nhalo || (nloc > 0 && (!local_node || !halo_slot)))
    return fail(h, OR_E_ARG, "set_halo: bad argument");
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, set_halo_impl, nloc, local_node, halo_slot, count_ke, nhalo);
}

int or_ecycle_spmd_buffer_bytes(or_ecycle* h, long long* bytes) {
  if (!h || !bytes) return OR_E_ARG;
  if (!h->finalized) return fail(h, OR_E_STATE, "spmd_buffer_bytes before finalize");
  const int nh = spmd_nhalo(h);
  if (nh < 0) return fail(h, OR_E_STATE, "spmd_buffer_bytes before set_halo");
  *bytes = (long long)(h->cfg.precision == OR_PREC_SPLIT ? halo_buffer_bytes<float>(nh) : halo_buffer_bytes<double>(nh));
  return OR_OK;
}

int or_ecycle_spmd_begin(or_ecycle* h, or_ecycle_time* t) {
  int rc = spmd_ready(h, false);
  if (rc) return rc;
  if (!t) return fail(h, OR_E_ARG, "spmd_begin: null time");
  return DISPATCH(h, spmd_begin_impl, t);
}

int or_ecycle_spmd_elements(or_ecycle* h, void* dev_buf) {
  int rc = spmd_ready(h, true);
  if (rc) return rc;
  if (!dev_buf) return fail(h, OR_E_ARG, "spmd_elements: null buffer");
  return DISPATCH(h, spmd_elements_impl, dev_buf);
}

int or_ecycle_spmd_nodes(or_ecycle* h, const void* dev_bufs, int nranks) {
  int rc = spmd_ready(h, true);
  if (rc) return rc;
  if (!dev_bufs || nranks < 1) return fail(h, OR_E_ARG, "spmd_nodes: bad argument");
  return DISPATCH(h, spmd_nodes_impl, dev_bufs, nranks);
}

int or_ecycle_spmd_end(or_ecycle* h, or_ecycle_time* t) {
  int rc = spmd_ready(h, true);
  if (rc) return rc;
  if (!t) return fail(h, OR_E_ARG, "spmd_end: null time");
  return DISPATCH(h, spmd_end_impl, t);
}

int or_ecycle_get_nodes(or_ecycle* h, int part, double* x, double* d, double* v, double* vr) {
  if (!h || !h->finalized || part < 0 || part >= (int)h->parts.size()) return h ? fail(h, OR_E_ARG, "get_nodes") : OR_E_ARG;
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, get_nodes_impl, part, x, d, v, vr);
}

int or_ecycle_set_nodes(or_ecycle* h, int part, const double* x, const double* d, const double* v, const double* vr) {
  if (!h || !h->finalized || part < 0 || part >= (int)h->parts.size()) return h ? fail(h, OR_E_ARG, "set_nodes") : OR_E_ARG;
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, set_nodes_impl, part, x, d, v, vr);
}

int or_ecycle_get_hex_state(or_ecycle* h, int group, double* sig, double* eint, double* rho, double* qvis, double* pla,
                            double* epsd) {
  if (!h || !h->finalized || group < 0 || group >= (int)h->hex.size()) return h ? fail(h, OR_E_ARG, "get_hex_state") : OR_E_ARG;
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, hex_state_impl, group, sig, eint, rho, qvis, pla, epsd);
}

int or_ecycle_set_hex_state(or_ecycle* h, int group, const double* sig, const double* eint, const double* rho,
                            const double* qvis, const double* pla, const double* epsd) {
  if (!h || !h->finalized || group < 0 || group >= (int)h->hex.size()) return h ? fail(h, OR_E_ARG, "set_hex_state") : OR_E_ARG;
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, set_hex_state_impl, group, sig, eint, rho, qvis, pla, epsd);
}

int or_ecycle_set_shell_state(or_ecycle* h, int group, const double* sig, const double* pla, const double* thk,
                              const double* hourg, const double* eint) {
  if (!h || !h->finalized || group < 0 || group >= (int)h->shell.size())
    return h ? fail(h, OR_E_ARG, "set_shell_state") : OR_E_ARG;
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, set_shell_state_impl, group, sig, pla, thk, hourg, eint);
}

int or_ecycle_set_energy_sums(or_ecycle* h, int part, double hourglass, double plastic_work, double external_work) {
  if (!h || part < 0 || part >= (int)h->parts.size()) return h ? fail(h, OR_E_ARG, "set_energy_sums") : OR_E_ARG;
  HPart& P = h->parts[part];
  P.ehour0 = hourglass; P.wpla0 = plastic_work; P.wext0 = external_work;
  return OR_OK;
}

int or_ecycle_get_shell_state(or_ecycle* h, int group, double* sig, double* pla, double* thk, double* hourg,
                              double* eint) {
  if (!h || !h->finalized || group < 0 || group >= (int)h->shell.size())
    return h ? fail(h, OR_E_ARG, "get_shell_state") : OR_E_ARG;
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, shell_state_impl, group, sig, pla, thk, hourg, eint);
}

int or_ecycle_energies(or_ecycle* h, int part, or_energies* e) {
  if (!h || !h->finalized || !e || part < 0 || part >= (int)h->parts.size()) return h ? fail(h, OR_E_ARG, "energies") : OR_E_ARG;
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, energies_impl, part, e);
}

int or_ecycle_error_info(or_ecycle* h, int* code, int* index) {
  if (!h || !code || !index) return OR_E_ARG;
  *code = h->last_code;
  *index = h->last_index;
  return OR_OK;
}

int or_ecycle_phase_times(or_ecycle* h, double* ms4) {
  if (!h || !ms4) return OR_E_ARG;
  for (int i = 0; i < 4; ++i) ms4[i] = h->phase_ms[i];
  return OR_OK;
}

int or_ecycle_kernel_times(or_ecycle* h, int reps, double* us3) {
  Trace tr("or_ecycle_kernel_times");
  if (!h || !us3) return OR_E_ARG;
  if (!h->finalized) return fail(h, OR_E_STATE, "kernel_times before finalize");
  if (reps <= 0 || reps > 4096) return fail(h, OR_E_ARG, "kernel_times: reps outside 1..4096");
  cudaSetDevice(h->cfg.device);
  return DISPATCH(h, kernel_times_impl, reps, us3);
}

int or_ecycle_launch_count(or_ecycle* h, long long* n) {
  if (!h || !n) return OR_E_ARG;
  *n = h->launches;
  return OR_OK;
}

int or_ecycle_stream(or_ecycle* h, void** stream) {
  if (!h || !stream) return OR_E_ARG;
  *stream = (void*)h->stream;
  return OR_OK;
}

int or_ecycle_device_bytes(or_ecycle* h, long long* bytes) {
  if (!h || !bytes) return OR_E_ARG;
  *bytes = h->dev_bytes;
  return OR_OK;
}

int or_ecycle_persistent_info(or_ecycle* h, int* on, int* ctas, int* threads) {
  if (!h || !on) return OR_E_ARG;
  if (!h->finalized) return fail(h, OR_E_STATE, "persistent_info before finalize");
  int g = 0, t = 0, o = 0;
  if (h->cfg.precision == OR_PREC_SPLIT) {
    const auto& q = ((Impl<float>*)h->impl)->per;
    o = q.on; g = q.G; t = q.T;
  } else {
    const auto& q = ((Impl<double>*)h->impl)->per;
    o = q.on; g = q.G; t = q.T;
  }
  *on = o;
  if (ctas) *ctas = o ? g : 0;
  if (threads) *threads = o ? t : 0;
  return OR_OK;
}

}  // extern "C"
