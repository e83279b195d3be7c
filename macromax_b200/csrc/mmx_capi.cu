// C ABI of macromax_b200: plans, launch configuration and the extern "C" entry points declared in
// include/macromax_b200.h.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "mmx_fast.cuh"
#include "mmx_reg.cuh"
#include "mmx_plane.cuh"
#include "mmx_epro.cuh"
#include "mmx_magnetic.cuh"
#include "mmx_fftr.cuh"
#include "mmx_tma.cuh"
#include "mmx_modes.cuh"
#include "mmx_magpass.cuh"

#include <cudaTypedefs.h>

#define MMX_ABI_VERSION 1

static_assert(sizeof(mmx_rhs_state) == 112, "mmx_rhs_state layout is part of the ABI");

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(MMX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define MMX_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

constexpr size_t kSmemCap = 220 * 1024;

// Pass kernels are launched with programmatic stream serialization (the next pass may be scheduled while the
// previous one drains; the kernels wait for their predecessor's memory, see pdl_wait).  MMX_NO_PDL=1 turns it off.
bool pdl_enabled() {
  static const bool on = [] {
    const char* v = getenv("MMX_NO_PDL");
    return !(v && v[0] == '1');
  }();
  return on;
}

template <class... KArgs, class... Args>
cudaError_t launch_pass(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                        Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

// Raise a kernel's dynamic shared-memory limit once per device.  `configured` is the calling launcher's own static
// (one launcher per kernel instantiation) holding one bit per device ordinal; concurrent first calls may both set
// the attribute, which is harmless.
int allow_smem_once(std::atomic<uint64_t>& configured, const void* kern, int bytes) {
  int dev = 0;
  MMX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(MMX_ERR_ARG, "device ordinals above 63 are not supported");
  const uint64_t bit = 1ull << dev;
  if (!(configured.load(std::memory_order_acquire) & bit)) {
    MMX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    configured.fetch_or(bit, std::memory_order_release);
  }
  return MMX_OK;
}

struct PassCfg {
  int axis;
  int ops;
  int64_t outer, inner;
  int P, sP, threads;
  size_t smem;
  int64_t tiles;
  int fast = 0;  // 1: compile-time specialised kernel (complex64, N in the specialised set)
  int reg = 0;   // 1: register-staged strided pass (k_reg_pass, 16-pencil tiles)
  int regc = 0;  // 1: register-staged contiguous prologue/epilogue pass (k_regc_pass) for an isotropic chi
  int pipe = 0;  // 1: persistent double-buffered variant of the same pass (k_pipe_pass)
  int plane = 0; // 1: plane pass over the two inner axes of a 3D grid (k_plane_pass), 2-CTA clusters
  int epro = 0;  // 1: epilogue fused with the next iteration's speculative prologue (k_regc_epro, k_regc_aniso_epro)
  int repair = 0;  // 1: prologue again for rejected right-hand sides (k_regc_repair)
  int regc_aniso = 0;  // 1: register-staged contiguous pass for a 3x3 chi (k_regc_aniso_pass), rc_tiles / rc_smem
  int csplit = 0;      // > 1: a strided FFT-only pass of a vector field run as csplit one-component CTAs per tile
  int64_t rc_tiles = 0;
  size_t rc_smem = 0;
  int tma = 0;        // 1: strided pass staged by bulk tensor copies (k_tma_pass) through `tmap`
  CUtensorMap tmap;   // 5-D map of the work buffer [B][C][outer][N][inner], box 16 x N x 1 x C x 1
};

bool reg_length(int n, int C) { return C == 3 ? (n == 64 || n == 128) : (n == 64 || n == 128 || n == 256 || n == 512); }
// the strided (middle) passes also take 192-sample vector pencils
bool reg_strided_length(int n, int C) { return reg_length(n, C) || (C == 3 && n == 192); }

constexpr int kFastP = 8;
bool fast_length(int n) { return n == 64 || n == 128 || n == 192 || n == 256 || n == 384 || n == 512; }

}  // namespace

struct mmx_plan {
  int device = 0;
  int ndim = 0;
  int64_t shape[3] = {1, 1, 1};
  int ncomp = 1;
  int batch = 1;
  int prec = MMX_C64;
  int64_t N = 1;
  FFTAxis ax[3];           // radix plans; tw points at device twiddles of the plan precision
  void* tw_dev[3] = {nullptr, nullptr, nullptr};
  void* kv_dev = nullptr;  // k tables, plan precision, concatenated
  int kv_off[3] = {0, 0, 0};
  bool kv_set = false;
  void* work = nullptr;    // T [batch][ncomp][N]
  double* partials = nullptr;
  int64_t partials_len = 0;
  unsigned int* done = nullptr;  // per-RHS tile counters of the epilogue pass (zero between iterations)
  std::vector<PassCfg> iter_passes;
  std::vector<PassCfg> defect_passes;
  bool force_generic = false;  // MMX_FORCE_GENERIC=1: use only the runtime-length kernels (tests)
  bool no_reg = false;         // MMX_NO_REG=1: shared-memory staged kernels for the strided passes (tests)
  bool pipe = false;           // MMX_PIPE=1: persistent double-buffered prologue/epilogue passes
  // polls of k_pipe_pass's staged-input waits before it loads the tile from global memory instead and raises
  // MMX_STATUS_TIMEOUT (MMX_PIPE_POLL_LIMIT, 0 .. 2^20: a test of that path; draining waits keep 2^20)
  int poll_limit = 1 << 20;
  bool plane = false;          // plane passes over the two inner axes (3D, 128 x 128 planes, isotropic chi)
  std::vector<PassCfg> plane_passes;  // the 3-pass schedule used when `plane` is set and chi is isotropic
  bool epro = false;           // fuse each epilogue with the next iteration's prologue
  bool tma = false;            // strided 128-sample passes staged by bulk tensor copies (k_tma_pass)
  bool wide_green = false;     // MMX_WIDE_GREEN=1: 16-pencil tiles for the vector axis-0 pass (tests)
  std::vector<PassCfg> epro_passes;   // [middle passes..., EPI+PRO, repair]; the first PRO runs once per call
  // The last iteration call on this plan whose fused epilogue left the next iteration's first pass (the prologue
  // and the contiguous-axis forward transform of the current field) in `work`, and its buffers: E0, E1, chi, src,
  // state.  mmx_iterate_graph_continue starts a chunk with the middle passes only when its buffers match.
  bool cont_valid = false;
  const void* cont_buf[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int cont_kind = 0;
  // L2 residency of the work buffer (MMX_L2_PERSIST=1): the middle passes re-read T from L2
  bool l2_persist = false;
  size_t l2_window = 0;
  size_t l2_prev_limit = 0;
};

namespace {

// Captured iteration chunks: one executable graph per (plans, buffers, iteration count).
struct GraphKey {
  std::vector<const void*> ptrs;  // plans and buffers
  std::vector<int> ints;          // chi kinds, iteration count
  bool operator==(const GraphKey& o) const { return ptrs == o.ptrs && ints == o.ints; }
};
struct GraphEntry {
  GraphKey key;
  cudaGraphExec_t exec;
};
std::mutex g_graph_mutex;
std::vector<GraphEntry> g_graphs;

void drop_graphs_of(const mmx_plan* p) {
  std::lock_guard<std::mutex> lock(g_graph_mutex);
  for (size_t i = 0; i < g_graphs.size();) {
    bool uses = false;
    for (const void* q : g_graphs[i].key.ptrs) uses |= (q == (const void*)p);
    if (uses) {
      cudaGraphExecDestroy(g_graphs[i].exec);
      g_graphs.erase(g_graphs.begin() + i);
    } else {
      ++i;
    }
  }
}

}  // namespace

namespace {

bool factorize(int n, FFTAxis& ax) {
  ax.n = n;
  ax.nst = 0;
  int m = n;
  const int pref[] = {8, 4, 2, 3, 5, 7, 11, 13};
  while (m > 1) {
    bool found = false;
    for (int r : pref) {
      if (m % r == 0) {
        if (ax.nst >= MMX_MAX_STAGES) return false;
        ax.radix[ax.nst++] = r;
        m /= r;
        found = true;
        break;
      }
    }
    if (!found) return false;
  }
  return true;
}

size_t word_bytes(int prec) { return prec == MMX_C128 ? 16 : 8; }

// Pencils per tile: as many as fit ~64 KB of shared memory (at least 4 consecutive strided pencils, i.e. one
// 32-byte sector per row, when the row fits), bounded by the 512-thread launch bound of the pass kernels.
// min_tiles > 0: narrow the tile (down to 4 pencils on a strided axis, 1 on the contiguous one) until the pass has
// at least that many tiles, so that small transforms still spread over the SMs
void choose_tile(const FFTAxis& ax, int C, int64_t outer, int64_t inner, int prec, PassCfg& pc,
                 int64_t min_tiles = 0) {
  const size_t wb = word_bytes(prec);
  const size_t budget = 64 * 1024;
  const int64_t npenc = outer * inner;
  int P = 1;
  auto smem_of = [&](int p) { return (size_t)C * ax.n * (size_t)(p > 1 ? p + 1 : 1) * wb; };
  auto thr_of = [&](int p) { return fft_tile_threads(C, p, ax); };
  const int pmax = (int)std::min<int64_t>(npenc, 64);
  if (inner > 1) {
    const int pmin = (int)std::min<int64_t>(inner, prec == MMX_C128 ? 2 : 4);
    P = pmin;
    while (P * 2 <= pmax && P * 2 <= inner && smem_of(P * 2) <= budget && thr_of(P * 2) <= 512) P *= 2;
    while (P > 1 && (smem_of(P) > kSmemCap || thr_of(P) > 512)) P /= 2;
  } else {
    P = 1;
    while (P * 2 <= pmax && smem_of(P * 2) <= budget && thr_of(P * 2) <= 512) P *= 2;
  }
  const int pfloor = inner > 1 ? (int)std::min<int64_t>(inner, 4) : 1;
  while (min_tiles > 0 && P / 2 >= pfloor && (npenc + P - 1) / P < min_tiles) P /= 2;
  pc.P = P;
  pc.sP = P > 1 ? P + 1 : 1;
  int thr = thr_of(P);
  thr = ((thr + 31) / 32) * 32;
  if (thr < 64) thr = 64;
  pc.threads = thr;
  pc.smem = smem_of(P);
  pc.tiles = (npenc + P - 1) / P;
  pc.outer = outer;
  pc.inner = inner;
}

template <class R, int C, int CHI, int OPS>
int launch_iter(const PassCfg& pc, IterArgs<R> a, int batch, cudaStream_t s) {
  auto kern = k_iter_pass<R, C, CHI, OPS>;
  static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
  {
    const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
    if (rc_ != MMX_OK) return rc_;
  }
  a.outer = pc.outer;
  a.inner = pc.inner;
  a.P = pc.P;
  a.sP = pc.sP;
  dim3 grid((unsigned)pc.tiles, (unsigned)batch);
  kern<<<grid, pc.threads, pc.smem, s>>>(a);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

template <class R, int C, int CHI>
int dispatch_ops(const PassCfg& pc, const IterArgs<R>& a, int batch, cudaStream_t s) {
  switch (pc.ops) {
    case OP_PRO | OP_FWD: return launch_iter<R, C, CHI, OP_PRO | OP_FWD>(pc, a, batch, s);
    case OP_FWD: return launch_iter<R, C, MMX_CHI_SCALAR, OP_FWD>(pc, a, batch, s);
    case OP_FWD | OP_G | OP_INV: return launch_iter<R, C, MMX_CHI_SCALAR, OP_FWD | OP_G | OP_INV>(pc, a, batch, s);
    case OP_INV: return launch_iter<R, C, MMX_CHI_SCALAR, OP_INV>(pc, a, batch, s);
    case OP_INV | OP_EPI: return launch_iter<R, C, CHI, OP_INV | OP_EPI>(pc, a, batch, s);
    case OP_PRO | OP_FWD | OP_G | OP_INV | OP_EPI:
      return launch_iter<R, C, CHI, OP_PRO | OP_FWD | OP_G | OP_INV | OP_EPI>(pc, a, batch, s);
    // defect pipeline (G^{-1})
    case OP_XLOAD | OP_FWD: return launch_iter<R, C, MMX_CHI_SCALAR, OP_XLOAD | OP_FWD>(pc, a, batch, s);
    case OP_FWD | OP_G | OP_GINV | OP_INV:
      return launch_iter<R, C, MMX_CHI_SCALAR, OP_FWD | OP_G | OP_GINV | OP_INV>(pc, a, batch, s);
    case OP_INV | OP_DEFECT: return launch_iter<R, C, CHI, OP_INV | OP_DEFECT>(pc, a, batch, s);
    case OP_XLOAD | OP_FWD | OP_G | OP_GINV | OP_INV | OP_DEFECT:
      return launch_iter<R, C, CHI, OP_XLOAD | OP_FWD | OP_G | OP_GINV | OP_INV | OP_DEFECT>(pc, a, batch, s);
    default: return fail(MMX_ERR_ARG, "internal: unknown pass operation set");
  }
}

template <int C, int CHI, int OPS, int N, bool STRIDED>
int launch_fast(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  auto kern = k_fast_pass<C, CHI, OPS, N, kFastP, STRIDED>;
  static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
  {
    const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
    if (rc_ != MMX_OK) return rc_;
  }
  a.outer = pc.outer;
  a.inner = pc.inner;
  a.P = kFastP;
  a.sP = kFastP + 1;
  dim3 grid((unsigned)pc.tiles, (unsigned)batch);
  if (a.l2_window) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(FastThreads<C, N, kFastP>::value);
    cfg.dynamicSmemBytes = pc.smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
    attr[0].val.accessPolicyWindow.base_ptr = (void*)a.T;
    attr[0].val.accessPolicyWindow.num_bytes = a.l2_window;
    attr[0].val.accessPolicyWindow.hitRatio = 1.0f;
    attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MMX_CUDA(cudaLaunchKernelEx(&cfg, kern, a));
  } else {
    MMX_CUDA(launch_pass(kern, grid, dim3(FastThreads<C, N, kFastP>::value), pc.smem, s, a));
  }
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

// 8-pencil tiles: the axis-0 pass (forward, Green multiply, inverse) of a vector field on 128-sample pencils
template <int C, int OPS, int N> constexpr bool kRegHalfTile = C == 3 && N == 128 && OPS == (OP_FWD | OP_G | OP_INV);

template <int C, int OPS, int N, int P>
int launch_reg_p(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  auto kern = k_reg_pass<C, OPS, N, P>;
  static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
  {
    const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
    if (rc_ != MMX_OK) return rc_;
  }
  a.outer = pc.outer;
  a.inner = pc.inner;
  a.P = P;
  a.sP = P;
  a.csplit = C == 1 ? pc.csplit : 0;
  dim3 grid((unsigned)pc.tiles, (unsigned)(batch * (a.csplit > 1 ? a.csplit : 1)));
  MMX_CUDA(launch_pass(kern, grid, dim3(RegThreads<C, N, P>::value), pc.smem, s, a));
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

template <int C, int OPS, int N>
int launch_reg(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  if constexpr ((C == 3 && N > 128 && N != 192) || (C == 1 && N == 192 && OPS == (OP_FWD | OP_G | OP_INV)) ||
                N == 384) {
    return fail(MMX_ERR_ARG, "internal: no register-staged kernel for this length");
  } else {
    if constexpr (kRegHalfTile<C, OPS, N>) {
      if (pc.P == 8) return launch_reg_p<C, OPS, N, 8>(pc, a, batch, s);
    }
    if (pc.P != kRegP) return fail(MMX_ERR_ARG, "internal: no register-staged kernel for this tile");
    auto kern = k_reg_pass<C, OPS, N>;
    static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
    {
      const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
      if (rc_ != MMX_OK) return rc_;
    }
    a.outer = pc.outer;
    a.inner = pc.inner;
    a.P = kRegP;
    a.sP = kRegP;
    a.csplit = C == 1 ? pc.csplit : 0;
    dim3 grid((unsigned)pc.tiles, (unsigned)(batch * (a.csplit > 1 ? a.csplit : 1)));
    MMX_CUDA(launch_pass(kern, grid, dim3(RegThreads<C, N>::value), pc.smem, s, a));
    MMX_CUDA(cudaGetLastError());
    return MMX_OK;
  }
}

int sm_count();

template <int C, int OPS, int N>
int launch_tma(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  if constexpr (N != 128) {
    return fail(MMX_ERR_ARG, "internal: no tensor-staged kernel for this length");
  } else {
    auto kern = k_tma_pass<C, OPS, N>;
    const size_t smem = mmx_tma::Layout<C, N>::bytes();
    static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
    {
      const int rc_ = allow_smem_once(configured, (const void*)kern, (int)smem);
      if (rc_ != MMX_OK) return rc_;
    }
    a.outer = pc.outer;
    a.inner = pc.inner;
    a.nrhs = batch;
    const int64_t tiles_per_rhs = pc.outer * pc.inner / kRegP;
    int per_sm = 1;  // resident CTAs per SM (two for the 3-component tiles; more for the scalar ones)
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, RegThreads<C, N>::value, smem) != cudaSuccess ||
        per_sm < 1) {
      cudaGetLastError();
      per_sm = 1;
    }
    const int64_t grid = std::min<int64_t>(tiles_per_rhs * batch, (int64_t)sm_count() * per_sm);
    MMX_CUDA(launch_pass(kern, dim3((unsigned)grid), dim3(RegThreads<C, N>::value), smem, s, a, pc.tmap,
                         (int)tiles_per_rhs));
    return MMX_OK;
  }
}

template <int C, int OPS, int N>
int launch_regc(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  if constexpr (N == 192 || N == 384 || (C == 3 && N > 128)) {
    return fail(MMX_ERR_ARG, "internal: no register-staged contiguous kernel for this length");
  } else {
    constexpr int PCK = (OPS & OP_EPI) ? RegCDefault<C, N>::PC_EPI : RegCDefault<C, N>::PC;
    auto kern = k_regc_pass<C, OPS, N, PCK>;
    static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
    {
      const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
      if (rc_ != MMX_OK) return rc_;
    }
    a.outer = pc.outer;
    a.inner = pc.inner;
    dim3 grid((unsigned)pc.rc_tiles, (unsigned)batch);
    MMX_CUDA(launch_pass(kern, grid, dim3(RegC<C, N, PCK>::THREADS), pc.rc_smem, s, a));
    MMX_CUDA(cudaGetLastError());
    return MMX_OK;
  }
}

template <int OPS, int N, int CHI>
int launch_regc_aniso(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  constexpr int PCK = RegCDefault<3, N>::PC;
  auto kern = k_regc_aniso_pass<OPS, N, PCK, CHI>;
  static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
  {
    const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
    if (rc_ != MMX_OK) return rc_;
  }
  a.outer = pc.outer;
  a.inner = pc.inner;
  dim3 grid((unsigned)pc.rc_tiles, (unsigned)batch);
  MMX_CUDA(launch_pass(kern, grid, dim3(RegC<3, N, PCK>::THREADS), pc.rc_smem, s, a));
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

// SM count of the current device, cached per device ordinal (0 .. 63)
int sm_count() {
  static std::atomic<int> cached[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  int n = cached[dev].load(std::memory_order_relaxed);
  if (n <= 0) {
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cached[dev].store(n, std::memory_order_relaxed);
  }
  return n;
}

template <int C, int OPS, int N>
int launch_pipe(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  if constexpr (N == 192 || N == 384 || (C == 3 && N > 128)) {
    return fail(MMX_ERR_ARG, "internal: no persistent kernel for this length");
  } else {
    constexpr int PCK = RegCDefault<C, N>::PC_PIPE;
    auto kern = k_pipe_pass<C, OPS, N, PCK>;
    const size_t smem = PipeLayout<C, OPS, N, PCK>::bytes();
    static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
    {
      const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
      if (rc_ != MMX_OK) return rc_;
    }
    const int64_t tiles_per_rhs = pc.outer / PCK;
    const int64_t ntiles = tiles_per_rhs * batch;
    int blocks_per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, RegC<C, N, PCK>::THREADS, smem);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
    const int64_t grid = std::min<int64_t>(ntiles, (int64_t)sm_count() * blocks_per_sm);
    a.nrhs = batch;
    kern<<<(unsigned)grid, RegC<C, N, PCK>::THREADS, smem, s>>>(a, (int)tiles_per_rhs);
    MMX_CUDA(cudaGetLastError());
    return MMX_OK;
  }
}

template <int C, int OPS>
int launch_plane(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  auto kern = k_plane_pass<C, OPS>;
  const size_t smem = mmx_plane::smem_bytes();
  static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
  {
    const int rc_ = allow_smem_once(configured, (const void*)kern, (int)smem);
    if (rc_ != MMX_OK) return rc_;
  }
  a.outer = pc.outer;
  a.inner = pc.inner;
  dim3 grid((unsigned)pc.tiles, (unsigned)batch);  // tiles = 2 n0 C (two CTAs per component plane)
  MMX_CUDA(launch_pass(kern, grid, dim3(mmx_plane::THREADS), smem, s, a));
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

template <int C, int N>
int launch_epro(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  if constexpr (N == 192 || N == 384 || (C == 3 && N > 128)) {
    return fail(MMX_ERR_ARG, "internal: no fused epilogue kernel for this length");
  } else {
    constexpr int PCK = RegCDefault<C, N>::PC_EPI;
    auto kern = k_regc_epro<C, N, PCK>;
    static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
    {
      const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
      if (rc_ != MMX_OK) return rc_;
    }
    a.outer = pc.outer;
    a.inner = pc.inner;
    a.nrhs = batch;
    dim3 grid((unsigned)pc.rc_tiles, (unsigned)batch);
    MMX_CUDA(launch_pass(kern, grid, dim3(RegC<C, N, PCK>::THREADS), pc.rc_smem, s, a));
    return MMX_OK;
  }
}

int sm_count();

template <int C, int N>
int launch_repair(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  if constexpr (N == 192 || N == 384 || (C == 3 && N > 128)) {
    return fail(MMX_ERR_ARG, "internal: no repair kernel for this length");
  } else {
    constexpr int PCK = RegCDefault<C, N>::PC;
    auto kern = k_regc_repair<C, N, PCK>;
    static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
    {
      const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
      if (rc_ != MMX_OK) return rc_;
    }
    a.outer = pc.outer;
    a.inner = pc.inner;
    a.nrhs = batch;
    // one CTA per SM: it only has work after a rejection, so the common, empty case should launch little
    const int64_t grid = std::min<int64_t>(pc.rc_tiles, (int64_t)sm_count());
    MMX_CUDA(launch_pass(kern, dim3((unsigned)grid), dim3(RegC<C, N, PCK>::THREADS), pc.rc_smem, s, a,
                         (int)pc.rc_tiles));
    return MMX_OK;
  }
}

// the fused epilogue / prologue and the repair pass for a 3x3 chi (k_regc_aniso_epro, k_regc_aniso_repair)
template <int N, int CHI>
int launch_aniso_epro(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  constexpr int PCK = RegCDefault<3, N>::PC;
  auto kern = k_regc_aniso_epro<N, PCK, CHI>;
  static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
  {
    const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
    if (rc_ != MMX_OK) return rc_;
  }
  a.outer = pc.outer;
  a.inner = pc.inner;
  a.nrhs = batch;
  dim3 grid((unsigned)pc.rc_tiles, (unsigned)batch);
  MMX_CUDA(launch_pass(kern, grid, dim3(RegC<3, N, PCK>::THREADS), pc.rc_smem, s, a));
  return MMX_OK;
}

template <int N, int CHI>
int launch_aniso_repair(const PassCfg& pc, IterArgs<float> a, int batch, cudaStream_t s) {
  constexpr int PCK = RegCDefault<3, N>::PC;
  auto kern = k_regc_aniso_repair<N, PCK, CHI>;
  static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
  {
    const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
    if (rc_ != MMX_OK) return rc_;
  }
  a.outer = pc.outer;
  a.inner = pc.inner;
  a.nrhs = batch;
  const int64_t grid = std::min<int64_t>(pc.rc_tiles, (int64_t)sm_count());
  MMX_CUDA(launch_pass(kern, dim3((unsigned)grid), dim3(RegC<3, N, PCK>::THREADS), pc.rc_smem, s, a,
                       (int)pc.rc_tiles));
  return MMX_OK;
}

template <int C, int CHI, int N>
int fast_ops(const PassCfg& pc, const IterArgs<float>& a, int batch, cudaStream_t s) {
  if (pc.epro || pc.repair) {
    if constexpr (CHI == MMX_CHI_SCALAR) {
      if (!pc.regc_aniso)
        return pc.epro ? launch_epro<C, N>(pc, a, batch, s) : launch_repair<C, N>(pc, a, batch, s);
    } else if constexpr (C == 3 && N == 192) {
      if (pc.regc_aniso)
        return pc.epro ? launch_aniso_epro<N, CHI>(pc, a, batch, s) : launch_aniso_repair<N, CHI>(pc, a, batch, s);
    }
    return fail(MMX_ERR_ARG, "internal: fused epilogue pass for another kind of chi");
  }
  if (pc.plane) {
    if constexpr (CHI == MMX_CHI_SCALAR && N == mmx_plane::N) {
      switch (pc.ops) {
        case OP_PRO | OP_FWD: return launch_plane<C, OP_PRO | OP_FWD>(pc, a, batch, s);
        case OP_INV | OP_EPI: return launch_plane<C, OP_INV | OP_EPI>(pc, a, batch, s);
        default: break;
      }
    }
    return fail(MMX_ERR_ARG, "internal: plane pass without a plane kernel");
  }
  if (pc.pipe && CHI == MMX_CHI_SCALAR) {
    switch (pc.ops) {
      case OP_PRO | OP_FWD: return launch_pipe<C, OP_PRO | OP_FWD, N>(pc, a, batch, s);
      case OP_INV | OP_EPI: return launch_pipe<C, OP_INV | OP_EPI, N>(pc, a, batch, s);
      default: break;
    }
  }
  if constexpr (CHI != MMX_CHI_SCALAR && C == 3 && N == 192) {
    if (pc.regc_aniso) {
      switch (pc.ops) {
        case OP_PRO | OP_FWD: return launch_regc_aniso<OP_PRO | OP_FWD, N, CHI>(pc, a, batch, s);
        case OP_INV | OP_EPI: return launch_regc_aniso<OP_INV | OP_EPI, N, CHI>(pc, a, batch, s);
        default: break;
      }
    }
  }
  if (pc.regc && CHI == MMX_CHI_SCALAR) {
    switch (pc.ops) {
      case OP_PRO | OP_FWD: return launch_regc<C, OP_PRO | OP_FWD, N>(pc, a, batch, s);
      case OP_INV | OP_EPI: return launch_regc<C, OP_INV | OP_EPI, N>(pc, a, batch, s);
      default: break;
    }
  }
  if (pc.tma) {
    switch (pc.ops) {
      case OP_FWD: return launch_tma<C, OP_FWD, N>(pc, a, batch, s);
      case OP_INV: return launch_tma<C, OP_INV, N>(pc, a, batch, s);
      case OP_FWD | OP_G | OP_INV: return launch_tma<C, OP_FWD | OP_G | OP_INV, N>(pc, a, batch, s);
      default: return fail(MMX_ERR_ARG, "internal: operation set without a tensor-staged kernel");
    }
  }
  if (pc.reg) {
    if (pc.csplit > 1) {  // one-component CTAs on a vector field (FFT-only passes)
      switch (pc.ops) {
        case OP_FWD: return launch_reg<1, OP_FWD, N>(pc, a, batch, s);
        case OP_INV: return launch_reg<1, OP_INV, N>(pc, a, batch, s);
        default: return fail(MMX_ERR_ARG, "internal: component split of a pass that mixes components");
      }
    }
    switch (pc.ops) {
      case OP_FWD: return launch_reg<C, OP_FWD, N>(pc, a, batch, s);
      case OP_INV: return launch_reg<C, OP_INV, N>(pc, a, batch, s);
      case OP_FWD | OP_G | OP_INV: return launch_reg<C, OP_FWD | OP_G | OP_INV, N>(pc, a, batch, s);
      default: return fail(MMX_ERR_ARG, "internal: operation set without a register-staged kernel");
    }
  }
  switch (pc.ops) {
    case OP_PRO | OP_FWD: return launch_fast<C, CHI, OP_PRO | OP_FWD, N, false>(pc, a, batch, s);
    case OP_INV | OP_EPI: return launch_fast<C, CHI, OP_INV | OP_EPI, N, false>(pc, a, batch, s);
    case OP_FWD: return launch_fast<C, MMX_CHI_SCALAR, OP_FWD, N, true>(pc, a, batch, s);
    case OP_INV: return launch_fast<C, MMX_CHI_SCALAR, OP_INV, N, true>(pc, a, batch, s);
    case OP_FWD | OP_G | OP_INV: return launch_fast<C, MMX_CHI_SCALAR, OP_FWD | OP_G | OP_INV, N, true>(pc, a, batch, s);
    default: return fail(MMX_ERR_ARG, "internal: operation set without a specialised kernel");
  }
}

template <int N>
int fast_dispatch_n(const PassCfg& pc, const IterArgs<float>& a, int C, int chi_kind, int batch, cudaStream_t s) {
  if (C == 1) return fast_ops<1, MMX_CHI_SCALAR, N>(pc, a, batch, s);
  if (chi_kind == MMX_CHI_SCALAR) return fast_ops<3, MMX_CHI_SCALAR, N>(pc, a, batch, s);
  if (chi_kind == MMX_CHI_SYM6) return fast_ops<3, MMX_CHI_SYM6, N>(pc, a, batch, s);
  return fast_ops<3, MMX_CHI_MAT3, N>(pc, a, batch, s);
}

int fast_dispatch(const PassCfg& pc, const IterArgs<float>& a, int C, int chi_kind, int batch, cudaStream_t s) {
  switch (a.ax.n) {
    case 64: return fast_dispatch_n<64>(pc, a, C, chi_kind, batch, s);
    case 128: return fast_dispatch_n<128>(pc, a, C, chi_kind, batch, s);
    case 192: return fast_dispatch_n<192>(pc, a, C, chi_kind, batch, s);
    case 256: return fast_dispatch_n<256>(pc, a, C, chi_kind, batch, s);
    case 384: return fast_dispatch_n<384>(pc, a, C, chi_kind, batch, s);
    case 512: return fast_dispatch_n<512>(pc, a, C, chi_kind, batch, s);
    default: return fail(MMX_ERR_ARG, "internal: no specialised kernel for this length");
  }
}

template <class R>
int dispatch_pass(const PassCfg& pc, const IterArgs<R>& a, int C, int chi_kind, int batch, cudaStream_t s) {
  if constexpr (std::is_same<R, float>::value) {
    if (pc.fast) {
      if (C == 1 && chi_kind != MMX_CHI_SCALAR) return fail(MMX_ERR_ARG, "a 3x3 chi needs a 3-component field");
      return fast_dispatch(pc, a, C, chi_kind, batch, s);
    }
  }
  if (C == 1) {
    if (chi_kind != MMX_CHI_SCALAR) return fail(MMX_ERR_ARG, "a 3x3 chi needs a 3-component field");
    return dispatch_ops<R, 1, MMX_CHI_SCALAR>(pc, a, batch, s);
  }
  if (chi_kind == MMX_CHI_SCALAR) return dispatch_ops<R, 3, MMX_CHI_SCALAR>(pc, a, batch, s);
  if (chi_kind == MMX_CHI_SYM6) return dispatch_ops<R, 3, MMX_CHI_SYM6>(pc, a, batch, s);
  return dispatch_ops<R, 3, MMX_CHI_MAT3>(pc, a, batch, s);
}

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    cudaGetLastError();
  });
  return fn;
}

// The tile map of a strided pass over the plan's work buffer T [B][C][outer][n][inner] (complex64 words as 8-byte
// elements): dimensions innermost first (inner, n, outer, C, B), box (16, n, 1, C, 1), the [c][j][pencil] tile of
// k_tma_pass.  False when the geometry does not qualify (the pass then keeps k_reg_pass).
bool encode_tile_map(const mmx_plan* p, int64_t outer, int n, int64_t inner, CUtensorMap* map) {
  auto enc = tensor_map_encoder();
  if (!enc || !p->work || inner % kRegP != 0 || n > 256 || p->ncomp > 256) return false;
  const cuuint64_t dims[5] = {(cuuint64_t)inner, (cuuint64_t)n, (cuuint64_t)outer, (cuuint64_t)p->ncomp,
                              (cuuint64_t)p->batch};
  const cuuint64_t strides[4] = {(cuuint64_t)inner * 8, (cuuint64_t)n * inner * 8, (cuuint64_t)p->N * 8,
                                 (cuuint64_t)p->ncomp * p->N * 8};
  const cuuint32_t box[5] = {(cuuint32_t)kRegP, (cuuint32_t)n, 1u, (cuuint32_t)p->ncomp, 1u};
  const cuuint32_t estr[5] = {1u, 1u, 1u, 1u, 1u};
  for (int i = 0; i < 4; ++i)
    if (strides[i] % 16 != 0) return false;
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_INT64, 5, p->work, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// pass sequence of one application of chi G chi (iteration) or of the FP64 defect
std::vector<PassCfg> build_passes(const mmx_plan* p, bool defect) {
  std::vector<PassCfg> v;
  const int d = p->ndim;
  auto geom = [&](int axis, int ops) {
    PassCfg pc;
    pc.axis = axis;
    pc.ops = ops;
    int64_t outer = 1, inner = 1;
    for (int i = 0; i < axis; ++i) outer *= p->shape[i];
    for (int i = axis + 1; i < d; ++i) inner *= p->shape[i];
    choose_tile(p->ax[axis], p->ncomp, outer, inner, p->prec, pc);
    const int n = (int)p->shape[axis];
    const bool ops_ok = !defect && d > 1;
    const bool geom_ok = inner > 1 ? (inner % kFastP == 0) : (outer % kFastP == 0);
    if (p->prec == MMX_C64 && fast_length(n) && ops_ok && geom_ok && !p->force_generic) {
      pc.fast = 1;
      pc.P = kFastP;
      pc.sP = kFastP + 1;
      pc.tiles = outer * inner / kFastP;
      pc.smem = ((size_t)p->ncomp * n * (kFastP + 1) + n) * sizeof(float2);
      pc.threads = 0;  // fixed by the specialisation
      const bool strided_op = ops == OP_FWD || ops == OP_INV || ops == (OP_FWD | OP_G | OP_INV);
      const bool contig_op = ops == (OP_PRO | OP_FWD) || ops == (OP_INV | OP_EPI);
      if (contig_op && inner == 1 && reg_length(n, p->ncomp) && !p->no_reg) {
        const bool epi = (ops & OP_EPI) != 0;
        int pcr = 1;
        switch (n * 4 + p->ncomp) {
          case 64 * 4 + 1: pcr = epi ? RegCDefault<1, 64>::PC_EPI : RegCDefault<1, 64>::PC; break;
          case 128 * 4 + 1: pcr = epi ? RegCDefault<1, 128>::PC_EPI : RegCDefault<1, 128>::PC; break;
          case 256 * 4 + 1: pcr = epi ? RegCDefault<1, 256>::PC_EPI : RegCDefault<1, 256>::PC; break;
          case 512 * 4 + 1: pcr = epi ? RegCDefault<1, 512>::PC_EPI : RegCDefault<1, 512>::PC; break;
          case 64 * 4 + 3: pcr = epi ? RegCDefault<3, 64>::PC_EPI : RegCDefault<3, 64>::PC; break;
          case 128 * 4 + 3: pcr = epi ? RegCDefault<3, 128>::PC_EPI : RegCDefault<3, 128>::PC; break;
        }
        int pcp = 1;
        switch (n * 4 + p->ncomp) {
          case 64 * 4 + 1: pcp = RegCDefault<1, 64>::PC_PIPE; break;
          case 128 * 4 + 1: pcp = RegCDefault<1, 128>::PC_PIPE; break;
          case 256 * 4 + 1: pcp = RegCDefault<1, 256>::PC_PIPE; break;
          case 512 * 4 + 1: pcp = RegCDefault<1, 512>::PC_PIPE; break;
          case 64 * 4 + 3: pcp = RegCDefault<3, 64>::PC_PIPE; break;
          case 128 * 4 + 3: pcp = RegCDefault<3, 128>::PC_PIPE; break;
        }
        if (outer % pcp == 0 && p->pipe) pc.pipe = 1;
        if (outer % pcr == 0) {
          pc.regc = 1;
          pc.rc_tiles = outer / pcr;
          pc.rc_smem = ((size_t)p->ncomp * pcr * (n + n / 16) + n) * sizeof(float2);
        }
      }
      if (contig_op && inner == 1 && n == 192 && p->ncomp == 3 && !p->no_reg) {
        // a 3x3 chi on 192-sample rows (the anisotropic 192^3 grids); an isotropic chi keeps k_fast_pass here
        constexpr int pca = RegCDefault<3, 192>::PC;
        if (outer % pca == 0) {
          pc.regc_aniso = 1;
          pc.rc_tiles = outer / pca;
          pc.rc_smem = ((size_t)3 * pca * (n + n / 16) + n) * sizeof(float2);
        }
      }
      if (strided_op && inner % kRegP == 0 && reg_strided_length(n, p->ncomp) && !p->no_reg) {
        pc.reg = 1;
        pc.P = kRegP;
        pc.sP = kRegP;
        pc.tiles = outer * inner / kRegP;
        pc.smem = ((size_t)p->ncomp * n * kRegP + n) * sizeof(float2);
        if (p->tma && n == 128 && encode_tile_map(p, outer, n, inner, &pc.tmap)) pc.tma = 1;
        if (!pc.tma && p->ncomp == 3 && (ops == OP_FWD || ops == OP_INV) && (n == 64 || n == 128 || n == 192)) {
          // The FFT-only strided passes of a vector field do not mix components: one-component CTAs, a third of
          // the work each, so the pass's last partial wave drains sooner (116.4 instead of 121.4 us per 128^3
          // vector iteration; the same registers, CTAs per SM and results).
          pc.csplit = 3;
          pc.smem = ((size_t)n * kRegP + n) * sizeof(float2);
        }
        if (!pc.tma && p->ncomp == 3 && ops == (OP_FWD | OP_G | OP_INV) && n == 128 && !p->wide_green) {
          // The vector axis-0 pass in 8-pencil tiles (192-thread CTAs, five per SM): half the work per CTA, so the
          // pass's last partial wave drains sooner, and more resident warps than two 384-thread CTAs.
          pc.P = pc.sP = 8;
          pc.tiles = outer * inner / 8;
          pc.smem = ((size_t)tile_rows<8>(3 * n) * 8 + n) * sizeof(float2);
        }
      }
    }
    v.push_back(pc);
  };
  const int first = defect ? (OP_XLOAD | OP_FWD) : (OP_PRO | OP_FWD);
  const int last = defect ? (OP_INV | OP_DEFECT) : (OP_INV | OP_EPI);
  const int mid = defect ? (OP_FWD | OP_G | OP_GINV | OP_INV) : (OP_FWD | OP_G | OP_INV);
  if (d == 1) {
    geom(0, first | last | mid);
    return v;
  }
  geom(d - 1, first);
  for (int a = d - 2; a >= 1; --a) geom(a, OP_FWD);
  geom(0, mid);
  for (int a = 1; a <= d - 2; ++a) geom(a, OP_INV);
  geom(d - 1, last);
  return v;
}

// The per-iteration passes with the epilogue fused to the next iteration's speculative prologue: the middle
// passes of the plain schedule, then [INV EPI + PRO FWD] and the repair pass (empty when the contiguous axis has no
// register-staged kernel).  The plain schedule's first pass runs once at the start of every chunk of iterations.
// The list serves an isotropic chi, or a 3x3 chi when its passes carry regc_aniso (epro_serves below).
std::vector<PassCfg> build_epro_passes(const mmx_plan* p) {
  std::vector<PassCfg> v;
  if (p->ndim < 2 || p->prec != MMX_C64 || p->force_generic) return v;
  const std::vector<PassCfg> plain = build_passes(p, false);
  if (plain.size() < 3) return v;
  // isotropic chi (k_regc_epro) or a 3x3 chi (k_regc_aniso_epro; the passes keep their regc_aniso flag)
  const bool iso = plain.front().regc && plain.back().regc && !plain.front().pipe && !plain.back().pipe;
  const bool aniso = plain.front().regc_aniso && plain.back().regc_aniso;
  if (!iso && !aniso) return v;
  for (size_t k = 1; k + 1 < plain.size(); ++k) v.push_back(plain[k]);
  PassCfg epi = plain.back();
  epi.regc = 0;
  epi.epro = 1;
  PassCfg rep = plain.front();
  rep.regc = 0;
  rep.repair = 1;
  v.push_back(epi);
  v.push_back(rep);
  return v;
}

// The 3-pass schedule [PRO FWD ax2 FWD ax1] [FWD G INV ax0] [INV ax1 INV ax2 EPI] of a 3D complex64 grid with
// 128 x 128 planes (empty when the grid does not qualify).  The axis-0 pass is the one of the 5-pass schedule.
std::vector<PassCfg> build_plane_passes(const mmx_plan* p) {
  std::vector<PassCfg> v;
  if (p->ndim != 3 || p->prec != MMX_C64 || p->force_generic || p->shape[1] != mmx_plane::N ||
      p->shape[2] != mmx_plane::N)
    return v;
  const std::vector<PassCfg> five = build_passes(p, false);
  if (five.size() != 5 || !five[2].fast) return v;
  PassCfg pro = five[0];
  pro.plane = 1;
  pro.regc = pro.pipe = pro.reg = 0;
  pro.fast = 1;
  pro.tiles = 2 * p->shape[0] * p->ncomp;
  PassCfg epi = five[4];
  epi.plane = 1;
  epi.regc = epi.pipe = epi.reg = 0;
  epi.fast = 1;
  epi.tiles = pro.tiles;
  v.push_back(pro);
  v.push_back(five[2]);
  v.push_back(epi);
  return v;
}

// whether the plan's fused-epilogue passes apply to this kind of chi
bool epro_serves(const mmx_plan* p, int chi_kind) {
  if (p->epro_passes.empty()) return false;
  return p->epro_passes.back().regc_aniso ? chi_kind != MMX_CHI_SCALAR : chi_kind == MMX_CHI_SCALAR;
}

template <class R> IterArgs<R> base_args(mmx_plan* p) {
  IterArgs<R> a;
  memset(&a, 0, sizeof(a));
  a.N = p->N;
  a.ndim = p->ndim;
  for (int i = 0; i < 3; ++i) {
    a.dims[i] = (int)p->shape[i];
    a.kv[i] = p->kv_dev ? (const R*)p->kv_dev + p->kv_off[i] : nullptr;
  }
  a.T = (cpx<R>*)p->work;
  a.partials = p->partials;
  a.done = p->done;
  a.l2_window = p->l2_persist ? p->l2_window : 0;
  a.inv_total = (R)(1.0 / (double)p->N);
  a.poll_limit = p->poll_limit;
  return a;
}

// whether run_iterations takes the fused-epilogue schedule for this plan and chi
bool epro_runs(const mmx_plan* p, int chi_kind) {
  if (p->prec != MMX_C64) return false;
  const bool plane = p->plane && chi_kind == MMX_CHI_SCALAR && !p->plane_passes.empty();
  return !plane && p->epro && epro_serves(p, chi_kind);
}

// record the buffers of an iteration call just launched on the stream (the record is cleared unless the call ran
// the fused-epilogue schedule; later calls on the stream run after it)
void note_iteration_call(mmx_plan* p, const void* E0, const void* E1, const void* chi, int chi_kind, const void* src,
                         const void* st) {
  p->cont_valid = epro_runs(p, chi_kind);
  const void* b[5] = {E0, E1, chi, src, st};
  for (int i = 0; i < 5; ++i) p->cont_buf[i] = b[i];
  p->cont_kind = chi_kind;
}

bool can_continue(const mmx_plan* p, const void* E0, const void* E1, const void* chi, int chi_kind, const void* src,
                  const void* st) {
  const void* b[5] = {E0, E1, chi, src, st};
  if (!p->cont_valid || p->cont_kind != chi_kind || !epro_runs(p, chi_kind)) return false;
  for (int i = 0; i < 5; ++i)
    if (p->cont_buf[i] != b[i]) return false;
  return true;
}

// `niter` iterations on stream s.  skip_first: the fused-epilogue schedule starts with the middle passes, because
// the previous call's last fused epilogue (or repair pass) already wrote this chunk's first pass to the work buffer.
template <class R>
int run_iterations(mmx_plan* p, void* E0, void* E1, const void* chi, int chi_kind, const void* src,
                   mmx_rhs_state* st, int niter, cudaStream_t s, bool skip_first = false) {
  IterArgs<R> a = base_args<R>(p);
  a.E0 = (cpx<R>*)E0;
  a.E1 = (cpx<R>*)E1;
  a.chi = (const cpx<R>*)chi;
  a.src = (const cpx<R>*)src;
  a.st = st;
  // the accept/reject decision is taken by the last tile of the epilogue pass (no separate launch)
  const bool plane = std::is_same<R, float>::value && p->plane && chi_kind == MMX_CHI_SCALAR &&
                     !p->plane_passes.empty();
  const bool epro = std::is_same<R, float>::value && !plane && p->epro && epro_serves(p, chi_kind);
  if (epro) {
    // first prologue of the chunk, then per iteration the middle passes, the fused epilogue + next prologue and
    // the repair pass
    int rc = MMX_OK;
    if (!skip_first) {
      a.ax = p->ax[p->iter_passes.front().axis];
      rc = dispatch_pass<R>(p->iter_passes.front(), a, p->ncomp, chi_kind, p->batch, s);
      if (rc != MMX_OK) return rc;
    }
    for (int it = 0; it < niter; ++it) {
      for (const PassCfg& pc : p->epro_passes) {
        a.ax = p->ax[pc.axis];
        rc = dispatch_pass<R>(pc, a, p->ncomp, chi_kind, p->batch, s);
        if (rc != MMX_OK) return rc;
      }
    }
    return MMX_OK;
  }
  const std::vector<PassCfg>& passes = plane ? p->plane_passes : p->iter_passes;
  for (int it = 0; it < niter; ++it) {
    for (const PassCfg& pc : passes) {
      a.ax = p->ax[pc.axis];
      int rc = dispatch_pass<R>(pc, a, p->ncomp, chi_kind, p->batch, s);
      if (rc != MMX_OK) return rc;
    }
  }
  return MMX_OK;
}

// Register-staged FFT-only pass (mmx_fftr.cuh) for one axis of mmx_fftn: false if this axis has none (then the
// runtime-radix pass runs).  Contiguous axis: PC rows per tile, the default tile when that gives two waves of tiles,
// else a quarter of it.
template <int DIR, int N>
bool fftr_axis_n(const float2* in, float2* out, int64_t outer, int64_t inner, const float2* tw, float scale,
                 cudaStream_t s, cudaError_t* err) {
  if (inner > 1) {
    if (inner % kRegP != 0 || scale != 1.0f) return false;
    const int64_t tiles = outer * inner / kRegP;
    const size_t smem = ((size_t)N * kRegP + N) * sizeof(float2);
    static std::atomic<uint64_t> configured{0};  // 512-sample tiles need more than the default 48 KiB
    if (allow_smem_once(configured, (const void*)k_fftr_strided<DIR, N>, (int)kSmemCap) != MMX_OK) {
      *err = cudaErrorInvalidValue;
      return true;
    }
    k_fftr_strided<DIR, N><<<(unsigned)tiles, RegThreads<1, N>::value, smem, s>>>(in, out, inner, tw);
    *err = cudaGetLastError();
    return true;
  }
  constexpr int PCB = RegCDefault<1, N>::PC;
  constexpr int PCS = PCB >= 4 ? PCB / 4 : 1;
  const int64_t rows = outer;
  if (rows % PCB == 0 && rows / PCB >= 2 * (int64_t)sm_count()) {
    const size_t smem = ((size_t)PCB * RegC<1, N, PCB>::PITCH + N) * sizeof(float2);
    k_fftr_contig<DIR, N, PCB><<<(unsigned)(rows / PCB), RegC<1, N, PCB>::THREADS, smem, s>>>(in, out, tw, scale);
  } else if (rows % PCS == 0) {
    const size_t smem = ((size_t)PCS * RegC<1, N, PCS>::PITCH + N) * sizeof(float2);
    k_fftr_contig<DIR, N, PCS><<<(unsigned)(rows / PCS), RegC<1, N, PCS>::THREADS, smem, s>>>(in, out, tw, scale);
  } else {
    return false;
  }
  *err = cudaGetLastError();
  return true;
}

template <int DIR>
bool fftr_axis(int n, const float2* in, float2* out, int64_t outer, int64_t inner, const float2* tw, float scale,
               cudaStream_t s, cudaError_t* err) {
  switch (n) {
    case 64: return fftr_axis_n<DIR, 64>(in, out, outer, inner, tw, scale, s, err);
    case 128: return fftr_axis_n<DIR, 128>(in, out, outer, inner, tw, scale, s, err);
    case 256: return fftr_axis_n<DIR, 256>(in, out, outer, inner, tw, scale, s, err);
    case 512: return fftr_axis_n<DIR, 512>(in, out, outer, inner, tw, scale, s, err);
    default: return false;
  }
}

template <class R> int run_fftn(mmx_plan* p, const void* in, void* out, int64_t nbatch, int inverse, cudaStream_t s) {
  const int d = p->ndim;
  const void* cur_in = in;
  // the inverse's 1 / N is applied once, by the first (contiguous-axis) pass: to its input in the register-staged
  // pass, to its output in the runtime-radix one
  for (int k = 0; k < d; ++k) {
    const int axis = d - 1 - k;  // contiguous axis first
    int64_t outer = nbatch, inner = 1;
    for (int i = 0; i < axis; ++i) outer *= p->shape[i];
    for (int i = axis + 1; i < d; ++i) inner *= p->shape[i];
    if constexpr (std::is_same<R, float>::value) {
      if (!p->force_generic) {
        const float sc = (inverse && k == 0) ? (float)(1.0 / (double)p->N) : 1.0f;
        cudaError_t e = cudaSuccess;
        const float2* tw = (const float2*)p->ax[axis].tw;
        const bool ran = inverse ? fftr_axis<+1>(p->ax[axis].n, (const float2*)cur_in, (float2*)out, outer, inner, tw,
                                                 sc, s, &e)
                                 : fftr_axis<-1>(p->ax[axis].n, (const float2*)cur_in, (float2*)out, outer, inner, tw,
                                                 sc, s, &e);
        if (ran) {
          if (e != cudaSuccess) return cuda_fail(e, "register-staged FFT pass");
          cur_in = out;
          continue;
        }
      }
    }
    PassCfg pc;
    choose_tile(p->ax[axis], 1, outer, inner, p->prec, pc, 2 * (int64_t)sm_count());
    FFTPassArgs<R> a;
    a.ax = p->ax[axis];
    a.outer = outer;
    a.inner = inner;
    a.P = pc.P;
    a.sP = pc.sP;
    a.in = (const cpx<R>*)cur_in;
    a.out = (cpx<R>*)out;
    a.scale = (R)((inverse && k == 0) ? 1.0 / (double)p->N : 1.0);
    if (inverse) {
      auto kern = k_fft_pass<R, +1>;
      MMX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemCap));
      kern<<<(unsigned)pc.tiles, pc.threads, pc.smem, s>>>(a);
    } else {
      auto kern = k_fft_pass<R, -1>;
      MMX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemCap));
      kern<<<(unsigned)pc.tiles, pc.threads, pc.smem, s>>>(a);
    }
    MMX_CUDA(cudaGetLastError());
    cur_in = out;
  }
  return MMX_OK;
}

int grid_blocks(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

extern "C" {

const char* mmx_last_error(void) { return g_last_error.c_str(); }

int mmx_version(void) { return MMX_ABI_VERSION; }

int mmx_plan_create(int ndim, const int64_t* shape, int ncomp, int batch, int precision, mmx_plan** out) {
  if (!out) return fail(MMX_ERR_ARG, "plan output pointer is NULL");
  *out = nullptr;
  if (ndim < 1 || ndim > 3) return fail(MMX_ERR_UNSUPPORTED, "grids of 1 to 3 axes are supported");
  if (!shape) return fail(MMX_ERR_ARG, "shape is NULL");
  if (ncomp != 1 && ncomp != 3) return fail(MMX_ERR_ARG, "ncomp must be 1 or 3");
  if (batch < 1 || batch > 65535) return fail(MMX_ERR_ARG, "batch must be in 1..65535");
  if (precision != MMX_C64 && precision != MMX_C128) return fail(MMX_ERR_ARG, "precision must be MMX_C64 or MMX_C128");
  mmx_plan* p = new mmx_plan();
  cudaGetDevice(&p->device);
  p->ndim = ndim;
  p->ncomp = ncomp;
  p->batch = batch;
  p->prec = precision;
  p->N = 1;
  for (int i = 0; i < ndim; ++i) {
    if (shape[i] < 1 || shape[i] > 16384) {
      delete p;
      return fail(MMX_ERR_UNSUPPORTED, "axis lengths must be in 1..16384");
    }
    p->shape[i] = shape[i];
    p->N *= shape[i];
    if (!factorize((int)shape[i], p->ax[i])) {
      delete p;
      return fail(MMX_ERR_UNSUPPORTED, "axis length " + std::to_string(shape[i]) +
                                           " has a prime factor above 13 (not supported)");
    }
  }
  for (int i = ndim; i < 3; ++i) p->shape[i] = 1;
  const size_t wb = word_bytes(precision);
  // twiddles exp(-2 pi i t / n), computed in FP64
  int kv_total = 0;
  for (int i = 0; i < ndim; ++i) {
    const int n = (int)shape[i];
    std::vector<double> twd(2 * (size_t)n);
    for (int t = 0; t < n; ++t) {
      const double ang = -2.0 * M_PI * (double)t / (double)n;
      twd[2 * t] = std::cos(ang);
      twd[2 * t + 1] = std::sin(ang);
    }
    cudaError_t e = cudaMalloc(&p->tw_dev[i], wb * n);
    if (e != cudaSuccess) {
      mmx_plan_destroy(p);
      return cuda_fail(e, "cudaMalloc(twiddles)");
    }
    if (precision == MMX_C128) {
      e = cudaMemcpy(p->tw_dev[i], twd.data(), wb * n, cudaMemcpyHostToDevice);
    } else {
      std::vector<float> twf(2 * (size_t)n);
      for (size_t k = 0; k < twf.size(); ++k) twf[k] = (float)twd[k];
      e = cudaMemcpy(p->tw_dev[i], twf.data(), wb * n, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
      mmx_plan_destroy(p);
      return cuda_fail(e, "cudaMemcpy(twiddles)");
    }
    p->ax[i].tw = p->tw_dev[i];
    p->kv_off[i] = kv_total;
    kv_total += n;
  }
  cudaError_t e = cudaMalloc(&p->kv_dev, (wb / 2) * (size_t)kv_total);
  if (e == cudaSuccess) e = cudaMemset(p->kv_dev, 0, (wb / 2) * (size_t)kv_total);
  if (e == cudaSuccess) e = cudaMalloc(&p->work, wb * (size_t)batch * ncomp * p->N);
  if (e != cudaSuccess) {
    mmx_plan_destroy(p);
    return cuda_fail(e, "cudaMalloc(plan buffers)");
  }
  {
    const char* fg = getenv("MMX_FORCE_GENERIC");
    p->force_generic = fg && fg[0] == '1';
    const char* nr = getenv("MMX_NO_REG");
    p->no_reg = nr && nr[0] == '1';
    const char* pp = getenv("MMX_PIPE");
    p->pipe = pp && pp[0] == '1';
    const char* wg = getenv("MMX_WIDE_GREEN");
    p->wide_green = wg && wg[0] == '1';
    const char* pl = getenv("MMX_PIPE_POLL_LIMIT");
    if (pl && pl[0]) p->poll_limit = std::max(0, std::min(1 << 20, atoi(pl)));
    const char* lp = getenv("MMX_L2_PERSIST");
    if (lp && lp[0] == '1' && precision == MMX_C64) {
      int maxp = 0, maxw = 0;
      cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, p->device);
      cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, p->device);
      const size_t tbytes = wb * (size_t)batch * ncomp * p->N;
      if (maxp > 0 && maxw > 0) {
        cudaDeviceGetLimit(&p->l2_prev_limit, cudaLimitPersistingL2CacheSize);
        const size_t want = std::min<size_t>((size_t)maxp, tbytes);
        if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) == cudaSuccess) {
          p->l2_persist = true;
          p->l2_window = std::min<size_t>(tbytes, (size_t)maxw);
        }
        cudaGetLastError();
      }
    }
  }
  p->iter_passes = build_passes(p, false);
  p->defect_passes = build_passes(p, true);
  p->plane_passes = build_plane_passes(p);
  p->epro_passes = build_epro_passes(p);
  int64_t maxt = 2048;  // enough partial sums for any tile width (at most one tile per pencil)
  for (int i = 0; i < ndim; ++i) maxt = std::max<int64_t>(maxt, p->N / shape[i]);
  p->partials_len = (int64_t)batch * maxt * 2;
  e = cudaMalloc(&p->partials, sizeof(double) * p->partials_len);
  if (e == cudaSuccess) e = cudaMalloc(&p->done, sizeof(unsigned int) * batch);
  if (e == cudaSuccess) e = cudaMemset(p->done, 0, sizeof(unsigned int) * batch);
  if (e != cudaSuccess) {
    mmx_plan_destroy(p);
    return cuda_fail(e, "cudaMalloc(partials)");
  }
  for (auto& pc : p->iter_passes) {
    if (pc.smem > kSmemCap || pc.threads > 512) {
      mmx_plan_destroy(p);
      return fail(MMX_ERR_UNSUPPORTED, "axis too long for the shared-memory FFT with this many components");
    }
  }
  *out = p;
  return MMX_OK;
}

int mmx_plan_destroy(mmx_plan* p) {
  if (!p) return MMX_OK;
  drop_graphs_of(p);
  for (int i = 0; i < 3; ++i)
    if (p->tw_dev[i]) cudaFree(p->tw_dev[i]);
  if (p->kv_dev) cudaFree(p->kv_dev);
  if (p->work) cudaFree(p->work);
  if (p->partials) cudaFree(p->partials);
  if (p->done) cudaFree(p->done);
  if (p->l2_persist) {  // hand the persisting set-aside back
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, p->l2_prev_limit);
    cudaGetLastError();
  }
  delete p;
  return MMX_OK;
}

int mmx_plan_set_kvectors(mmx_plan* p, const double* k) {
  if (!p || !k) return fail(MMX_ERR_ARG, "NULL plan or k");
  int total = 0;
  for (int i = 0; i < p->ndim; ++i) total += (int)p->shape[i];
  if (p->prec == MMX_C128) {
    MMX_CUDA(cudaMemcpy(p->kv_dev, k, sizeof(double) * total, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> kf(total);
    for (int i = 0; i < total; ++i) kf[i] = (float)k[i];
    MMX_CUDA(cudaMemcpy(p->kv_dev, kf.data(), sizeof(float) * total, cudaMemcpyHostToDevice));
  }
  p->kv_set = true;
  return MMX_OK;
}

int mmx_fftn(mmx_plan* p, const void* in, void* out, int64_t nbatch, int inverse, void* stream) {
  if (!p || !in || !out) return fail(MMX_ERR_ARG, "NULL plan or buffer");
  if (nbatch < 1) return fail(MMX_ERR_ARG, "nbatch must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  if (p->prec == MMX_C128) return run_fftn<double>(p, in, out, nbatch, inverse, s);
  return run_fftn<float>(p, in, out, nbatch, inverse, s);
}

int mmx_norm(mmx_plan* p, const void* x, int64_t nwords, int precision, double* out_dev, void* stream) {
  if (!p || !x || !out_dev) return fail(MMX_ERR_ARG, "NULL plan or buffer");
  if (nwords < 0) return fail(MMX_ERR_ARG, "negative size");
  cudaStream_t s = (cudaStream_t)stream;
  int blocks = grid_blocks(nwords, 256);
  if (blocks > p->partials_len) blocks = (int)p->partials_len;
  if (precision == MMX_C128)
    k_norm_partials<double><<<blocks, 256, 0, s>>>((const double2*)x, nwords, p->partials);
  else
    k_norm_partials<float><<<blocks, 256, 0, s>>>((const float2*)x, nwords, p->partials);
  MMX_CUDA(cudaGetLastError());
  k_norm_final<<<1, 256, 0, s>>>(p->partials, blocks, out_dev);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

int mmx_iterate(mmx_plan* p, void* E0, void* E1, const void* chi, int chi_kind, const void* src,
                mmx_rhs_state* state, int niter, void* stream) {
  if (!p || !E0 || !E1 || !chi || !src || !state) return fail(MMX_ERR_ARG, "NULL plan or buffer");
  if (chi_kind != MMX_CHI_SCALAR && chi_kind != MMX_CHI_MAT3 && chi_kind != MMX_CHI_SYM6)
    return fail(MMX_ERR_ARG, "unknown chi_kind");
  if (!p->kv_set) return fail(MMX_ERR_ARG, "k-vectors not set (mmx_plan_set_kvectors)");
  if (niter < 0) return fail(MMX_ERR_ARG, "negative iteration count");
  cudaStream_t s = (cudaStream_t)stream;
  p->cont_valid = false;
  const int rc = p->prec == MMX_C128 ? run_iterations<double>(p, E0, E1, chi, chi_kind, src, state, niter, s)
                                     : run_iterations<float>(p, E0, E1, chi, chi_kind, src, state, niter, s);
  if (rc == MMX_OK && niter > 0) note_iteration_call(p, E0, E1, chi, chi_kind, src, state);
  return rc;
}

int mmx_defect(mmx_plan* p, const void* x, const void* chi, int chi_kind, const void* src, const mmx_rhs_state* st,
               void* s_out, void* stream) {
  if (!p || !x || !chi || !src || !st || !s_out) return fail(MMX_ERR_ARG, "NULL plan or buffer");
  if (p->prec != MMX_C128) return fail(MMX_ERR_ARG, "mmx_defect needs a complex128 plan");
  if (!p->kv_set) return fail(MMX_ERR_ARG, "k-vectors not set (mmx_plan_set_kvectors)");
  cudaStream_t s = (cudaStream_t)stream;
  p->cont_valid = false;  // the defect transforms run in the work buffer
  IterArgs<double> a = base_args<double>(p);
  a.E0 = (double2*)x;
  a.E1 = (double2*)x;
  a.chi = (const double2*)chi;
  a.src = (const double2*)src;
  a.st = st;
  a.aux = (float2*)s_out;
  for (const PassCfg& pc : p->defect_passes) {
    a.ax = p->ax[pc.axis];
    int rc = dispatch_pass<double>(pc, a, p->ncomp, chi_kind, p->batch, s);
    if (rc != MMX_OK) return rc;
  }
  return MMX_OK;
}

int mmx_accumulate(void* x, const void* delta, int64_t nwords, void* stream) {
  if (!x || !delta) return fail(MMX_ERR_ARG, "NULL buffer");
  cudaStream_t s = (cudaStream_t)stream;
  k_accumulate<<<grid_blocks(nwords, 256), 256, 0, s>>>((double2*)x, (const float2*)delta, nwords);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

int mmx_adjoint_grad(const void* E, const void* nu, void* grad, int64_t batch, int ncomp, int64_t nvox,
                     int precision, double scale, void* stream) {
  if (!E || !nu || !grad) return fail(MMX_ERR_ARG, "NULL buffer");
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = grid_blocks(batch * nvox, 256);
  if (precision == MMX_C128)
    k_adjoint_grad<double><<<blocks, 256, 0, s>>>((const double2*)E, (const double2*)nu, (double2*)grad, batch, ncomp,
                                                  nvox, scale);
  else
    k_adjoint_grad<float><<<blocks, 256, 0, s>>>((const float2*)E, (const float2*)nu, (float2*)grad, batch, ncomp,
                                                 nvox, (float)scale);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

int mmx_pointwise_mul(const void* A, int ra, int ca, const void* B, int cb, int b_broadcast, void* out, int64_t nvox,
                      int precision, void* stream) {
  if (!A || !B || !out) return fail(MMX_ERR_ARG, "NULL buffer");
  if (ra < 1 || ca < 1 || cb < 1 || ra > 3 || ca > 3 || cb > 3) return fail(MMX_ERR_ARG, "matrix dims must be 1..3");
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = grid_blocks(nvox, 256);
  const int bstride = b_broadcast ? 0 : 1;
  if (precision == MMX_C128)
    k_pointwise_mul<double><<<blocks, 256, 0, s>>>((const double2*)A, ra, ca, (const double2*)B, cb, bstride,
                                                   (double2*)out, nvox);
  else
    k_pointwise_mul<float><<<blocks, 256, 0, s>>>((const float2*)A, ra, ca, (const float2*)B, cb, bstride,
                                                  (float2*)out, nvox);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

}  // extern "C"

namespace {

// Capture `niter` iterations of every plan into one graph: the plans' passes run on forked capture streams, so
// independent grids (e.g. batches of uneven sizes) become parallel branches of a single launch.
int capture_multi(int n, mmx_plan* const* plans, void* const* E0, void* const* E1, const void* const* chi,
                  const int* chi_kind, const void* const* src, mmx_rhs_state* const* st, int niter, bool skip_first,
                  cudaGraphExec_t* out) {
  std::vector<cudaStream_t> streams(n + 1, nullptr);
  std::vector<cudaEvent_t> events(n + 1, nullptr);
  int rc = MMX_OK;
  cudaGraph_t graph = nullptr;
  bool capturing = false;
  for (int i = 0; i <= n && rc == MMX_OK; ++i) {
    if (cudaStreamCreateWithFlags(&streams[i], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&events[i], cudaEventDisableTiming) != cudaSuccess)
      rc = fail(MMX_ERR_CUDA, "graph capture: stream/event creation failed");
  }
  if (rc == MMX_OK) {
    cudaError_t e = cudaStreamBeginCapture(streams[0], cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamBeginCapture");
    else capturing = true;
  }
  if (rc == MMX_OK) {
    cudaEventRecord(events[n], streams[0]);  // fork point
    for (int i = 0; i < n && rc == MMX_OK; ++i) {
      cudaStreamWaitEvent(streams[i + 1], events[n], 0);
      mmx_plan* p = plans[i];
      if (p->prec == MMX_C128)
        rc = run_iterations<double>(p, E0[i], E1[i], chi[i], chi_kind[i], src[i], st[i], niter, streams[i + 1]);
      else
        rc = run_iterations<float>(p, E0[i], E1[i], chi[i], chi_kind[i], src[i], st[i], niter, streams[i + 1],
                                   skip_first);
      cudaEventRecord(events[i], streams[i + 1]);
      cudaStreamWaitEvent(streams[0], events[i], 0);  // join
    }
  }
  if (capturing) {
    cudaError_t e = cudaStreamEndCapture(streams[0], &graph);
    if (rc == MMX_OK && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamEndCapture");
  }
  if (rc == MMX_OK) {
    cudaError_t e = cudaGraphInstantiate(out, graph, 0);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphInstantiate");
  }
  if (graph) cudaGraphDestroy(graph);
  for (int i = 0; i <= n; ++i) {
    if (events[i]) cudaEventDestroy(events[i]);
    if (streams[i]) cudaStreamDestroy(streams[i]);
  }
  cudaGetLastError();
  return rc;
}

}  // namespace

namespace {
// Find or capture the graph of `niter` iterations of the plans and launch it on `stream` (launch = false: capture
// and upload only).  cont (one plan): continue the previous call on these buffers -- the chunk starts with the middle
// passes when the plan's record says the work buffer holds its first pass (can_continue); a prepared call then
// captures that graph as well as the self-contained one.
int iterate_multi(int n, mmx_plan* const* plans, void* const* E0, void* const* E1, const void* const* chi,
                  const int* chi_kind, const void* const* src, mmx_rhs_state* const* state, int niter, void* stream,
                  bool launch, bool cont = false) {
  if (n < 1 || !plans || !E0 || !E1 || !chi || !chi_kind || !src || !state) return fail(MMX_ERR_ARG, "NULL argument");
  if (niter < 1) return fail(MMX_ERR_ARG, "niter must be positive");
  GraphKey key;
  for (int i = 0; i < n; ++i) {
    mmx_plan* p = plans[i];
    if (!p || !E0[i] || !E1[i] || !chi[i] || !src[i] || !state[i]) return fail(MMX_ERR_ARG, "NULL plan or buffer");
    if (chi_kind[i] != MMX_CHI_SCALAR && chi_kind[i] != MMX_CHI_MAT3 && chi_kind[i] != MMX_CHI_SYM6)
      return fail(MMX_ERR_ARG, "unknown chi_kind");
    if (!p->kv_set) return fail(MMX_ERR_ARG, "k-vectors not set (mmx_plan_set_kvectors)");
    key.ptrs.insert(key.ptrs.end(), {(const void*)p, E0[i], E1[i], chi[i], src[i], (const void*)state[i]});
    key.ints.push_back(chi_kind[i]);
  }
  key.ints.push_back(niter);
  const bool skip = cont && n == 1 && can_continue(plans[0], E0[0], E1[0], chi[0], chi_kind[0], src[0], state[0]);
  // a prepared continuation also captures the self-contained graph; a launch takes the one that applies
  for (int variant = (!launch && skip) ? 0 : (skip ? 1 : 0); variant <= (skip ? 1 : 0); ++variant) {
    GraphKey k = key;
    k.ints.push_back(variant);
    cudaGraphExec_t exec = nullptr;
    {
      std::lock_guard<std::mutex> lock(g_graph_mutex);
      for (const GraphEntry& g : g_graphs)
        if (g.key == k) exec = g.exec;
    }
    if (!exec) {
      const int rc = capture_multi(n, plans, E0, E1, chi, chi_kind, src, state, niter, variant == 1, &exec);
      if (rc != MMX_OK) return rc;
      {
        std::lock_guard<std::mutex> lock(g_graph_mutex);
        g_graphs.push_back(GraphEntry{k, exec});
      }
      if (!launch) {
        // a prepared graph is also uploaded now, so that its first launch does not pay for the upload
        MMX_CUDA(cudaGraphUpload(exec, (cudaStream_t)0));
        MMX_CUDA(cudaStreamSynchronize((cudaStream_t)0));
      }
    }
    if (launch) {
      for (int i = 0; i < n; ++i) plans[i]->cont_valid = false;
      MMX_CUDA(cudaGraphLaunch(exec, (cudaStream_t)stream));
      for (int i = 0; i < n; ++i) note_iteration_call(plans[i], E0[i], E1[i], chi[i], chi_kind[i], src[i], state[i]);
    }
  }
  return MMX_OK;
}
}  // namespace

extern "C" int mmx_iterate_multi(int n, mmx_plan* const* plans, void* const* E0, void* const* E1,
                                 const void* const* chi, const int* chi_kind, const void* const* src,
                                 mmx_rhs_state* const* state, int niter, void* stream) {
  return iterate_multi(n, plans, E0, E1, chi, chi_kind, src, state, niter, stream, true);
}

extern "C" int mmx_iterate_graph(mmx_plan* p, void* E0, void* E1, const void* chi, int chi_kind, const void* src,
                                 mmx_rhs_state* state, int niter, void* stream) {
  return iterate_multi(1, &p, &E0, &E1, &chi, &chi_kind, &src, &state, niter, stream, true);
}

extern "C" int mmx_iterate_graph_prepare(mmx_plan* p, void* E0, void* E1, const void* chi, int chi_kind,
                                         const void* src, mmx_rhs_state* state, int niter) {
  return iterate_multi(1, &p, &E0, &E1, &chi, &chi_kind, &src, &state, niter, nullptr, false, true);
}

extern "C" int mmx_iterate_graph_continue(mmx_plan* p, void* E0, void* E1, const void* chi, int chi_kind,
                                          const void* src, mmx_rhs_state* state, int niter, void* stream) {
  return iterate_multi(1, &p, &E0, &E1, &chi, &chi_kind, &src, &state, niter, stream, true, true);
}

extern "C" int mmx_plan_set_variant(mmx_plan* p, unsigned flags) {
  if (!p) return fail(MMX_ERR_ARG, "NULL plan");
  if (flags & ~63u) return fail(MMX_ERR_ARG, "unknown variant flags");
  drop_graphs_of(p);  // captured graphs hold the previous kernels
  p->cont_valid = false;
  p->force_generic = (flags & MMX_VARIANT_GENERIC) != 0;
  p->no_reg = (flags & MMX_VARIANT_SHARED_STAGED) != 0;
  p->pipe = (flags & MMX_VARIANT_PERSISTENT) != 0;
  p->plane = (flags & MMX_VARIANT_PLANE) != 0;
  p->epro = (flags & MMX_VARIANT_FUSED_EPILOGUE) != 0;
  p->tma = (flags & MMX_VARIANT_TMA) != 0;
  p->iter_passes = build_passes(p, false);
  p->defect_passes = build_passes(p, true);
  p->plane_passes = build_plane_passes(p);
  p->epro_passes = build_epro_passes(p);
  for (const auto* list : {&p->iter_passes, &p->plane_passes, &p->epro_passes})
    for (auto& pc : *list)
      if (2 * (int64_t)p->batch * pc.tiles > p->partials_len) return fail(MMX_ERR_ARG, "internal: partials too small");
  return MMX_OK;
}

extern "C" unsigned mmx_plan_get_variant(const mmx_plan* p) {
  if (!p) return 0u;
  return (p->force_generic ? MMX_VARIANT_GENERIC : 0u) | (p->no_reg ? MMX_VARIANT_SHARED_STAGED : 0u) |
         (p->pipe ? MMX_VARIANT_PERSISTENT : 0u) | (p->plane ? MMX_VARIANT_PLANE : 0u) |
         (p->epro ? MMX_VARIANT_FUSED_EPILOGUE : 0u) | (p->tma ? MMX_VARIANT_TMA : 0u);
}

extern "C" int mmx_mat3_extremes(mmx_plan* p, const void* M, int64_t nvox, int mode, double ab, double* out_dev,
                                 void* stream) {
  if (!p || !M || !out_dev) return fail(MMX_ERR_ARG, "NULL plan or buffer");
  if (mode != 0 && mode != 1) return fail(MMX_ERR_ARG, "mode must be 0 or 1");
  if (nvox < 1) return fail(MMX_ERR_ARG, "nvox must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  int blocks = grid_blocks(nvox, 256);
  if (2 * (int64_t)blocks > p->partials_len) blocks = (int)(p->partials_len / 2);
  k_mat3_extremes<<<blocks, 256, 0, s>>>((const double2*)M, nvox, mode, ab, p->partials);
  MMX_CUDA(cudaGetLastError());
  k_minmax_final<<<1, 256, 0, s>>>(p->partials, blocks, out_dev);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

namespace {
KGrid kgrid_of(const mmx_plan* p) {
  KGrid g;
  g.ndim = p->ndim;
  for (int i = 0; i < 3; ++i) g.dims[i] = (int)p->shape[i];
  g.N = p->N;
  return g;
}
template <class R> const R* kv_of(const mmx_plan* p, int axis) {
  return axis < p->ndim ? (const R*)p->kv_dev + p->kv_off[axis] : nullptr;
}
}  // namespace

extern "C" int mmx_curl_ft(mmx_plan* p, const void* F, void* out, void* stream) {
  if (!p || !F || !out) return fail(MMX_ERR_ARG, "NULL plan or buffer");
  if (!p->kv_set) return fail(MMX_ERR_ARG, "k-vectors not set (mmx_plan_set_kvectors)");
  if (F == out) return fail(MMX_ERR_ARG, "mmx_curl_ft cannot run in place");
  cudaStream_t s = (cudaStream_t)stream;
  const KGrid g = kgrid_of(p);
  const int blocks = grid_blocks(p->N, 256);
  if (p->prec == MMX_C128)
    k_curl_ft<double><<<blocks, 256, 0, s>>>((const double2*)F, (double2*)out, g, kv_of<double>(p, 0),
                                             kv_of<double>(p, 1), kv_of<double>(p, 2));
  else
    k_curl_ft<float><<<blocks, 256, 0, s>>>((const float2*)F, (float2*)out, g, kv_of<float>(p, 0),
                                            kv_of<float>(p, 1), kv_of<float>(p, 2));
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

extern "C" int mmx_green_ft(mmx_plan* p, void* F, double alpha_re, double alpha_im, void* stream) {
  if (!p || !F) return fail(MMX_ERR_ARG, "NULL plan or buffer");
  if (!p->kv_set) return fail(MMX_ERR_ARG, "k-vectors not set (mmx_plan_set_kvectors)");
  if (!(alpha_im > 0.0)) return fail(MMX_ERR_ARG, "alpha must have a positive imaginary part");
  cudaStream_t s = (cudaStream_t)stream;
  const KGrid g = kgrid_of(p);
  const int blocks = grid_blocks(p->N, 256);
  if (p->prec == MMX_C128)
    k_green_ft<double><<<blocks, 256, 0, s>>>((double2*)F, g, kv_of<double>(p, 0), kv_of<double>(p, 1),
                                              kv_of<double>(p, 2), alpha_re, alpha_im, nullptr);
  else
    k_green_ft<float><<<blocks, 256, 0, s>>>((float2*)F, g, kv_of<float>(p, 0), kv_of<float>(p, 1),
                                             kv_of<float>(p, 2), (float)alpha_re, (float)alpha_im, nullptr);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

extern "C" int mmx_chi_mix(const void* x, const void* d, const void* chi_ee, const void* chi_eh, const void* chi_he,
                           const void* chi_hh, const double* coef, void* u, void* w, int64_t nvox, int precision,
                           void* stream) {
  if (!x || !d || !chi_ee || !chi_eh || !chi_he || !chi_hh || !coef || !u || !w)
    return fail(MMX_ERR_ARG, "NULL buffer");
  if (nvox < 1) return fail(MMX_ERR_ARG, "nvox must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = grid_blocks(nvox, 256);
  if (precision == MMX_C128) {
    auto c = [&](int i) { return make_double2(coef[2 * i], coef[2 * i + 1]); };
    k_chi_mix<double><<<blocks, 256, 0, s>>>((const double2*)x, (const double2*)d, (const double2*)chi_ee,
                                             (const double2*)chi_eh, (const double2*)chi_he, (const double2*)chi_hh,
                                             c(0), c(1), c(2), c(3), c(4), (double2*)u, (double2*)w, nvox, nullptr);
  } else {
    auto c = [&](int i) { return make_float2((float)coef[2 * i], (float)coef[2 * i + 1]); };
    k_chi_mix<float><<<blocks, 256, 0, s>>>((const float2*)x, (const float2*)d, (const float2*)chi_ee,
                                            (const float2*)chi_eh, (const float2*)chi_he, (const float2*)chi_hh,
                                            c(0), c(1), c(2), c(3), c(4), (float2*)u, (float2*)w, nvox, nullptr);
  }
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

extern "C" int mmx_axpby(void* out, const void* x, const void* y, double a_re, double a_im, double b_re, double b_im,
                         int64_t nwords, int precision, void* stream) {
  if (!out || !x || !y) return fail(MMX_ERR_ARG, "NULL buffer");
  if (nwords < 1) return fail(MMX_ERR_ARG, "nwords must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = grid_blocks(nwords, 256);
  if (precision == MMX_C128)
    k_axpby<double><<<blocks, 256, 0, s>>>((double2*)out, (const double2*)x, (const double2*)y,
                                           make_double2(a_re, a_im), make_double2(b_re, b_im), nwords);
  else
    k_axpby<float><<<blocks, 256, 0, s>>>((float2*)out, (const float2*)x, (const float2*)y,
                                          make_float2((float)a_re, (float)a_im), make_float2((float)b_re, (float)b_im),
                                          nwords);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

namespace {
// ---- fused pass schedule for magnetic media (mmx_magpass.cuh), 2D and 3D grids ----
struct MagPass {
  int mode;
  int axis;
  PassCfg pc;
};

std::vector<MagPass> build_mag_passes(const mmx_plan* p) {
  std::vector<MagPass> v;
  const int d = p->ndim;
  if (d < 2 || d > 3) return v;
  auto add = [&](int mode, int axis, int C) {
    MagPass mp;
    mp.mode = mode;
    mp.axis = axis;
    int64_t outer = 1, inner = 1;
    for (int i = 0; i < axis; ++i) outer *= p->shape[i];
    for (int i = axis + 1; i < d; ++i) inner *= p->shape[i];
    // small grids (the reference's 2D magnetic cases) have few pencils: ask for at least two tiles per SM
    choose_tile(p->ax[axis], C, outer, inner, p->prec, mp.pc, 2 * (int64_t)sm_count());
    mp.pc.axis = axis;
    v.push_back(mp);
  };
  const int last = d - 1;
  add(MAG_E_FWD, last, 3);
  if (d == 3) add(MAG_MID_FWD3, 1, 3);
  add(MAG_K_CURL_E, 0, 3);
  if (d == 3) add(MAG_MID_INV3, 1, 3);
  add(MAG_MIX1, last, 6);
  if (d == 3) add(MAG_MID_FWD6, 1, 6);
  add(MAG_K_GREEN, 0, 6);
  if (d == 3) add(MAG_MID_INV6, 1, 6);
  add(MAG_MIX2, last, 6);
  if (d == 3) add(MAG_MID_FWD3, 1, 3);
  add(MAG_K_CURL, 0, 3);
  if (d == 3) add(MAG_MID_INV3, 1, 3);
  add(MAG_UPDATE, last, 3);
  for (const MagPass& mp : v)
    if (2 * mp.pc.tiles > p->partials_len || mp.pc.smem > kSmemCap) return std::vector<MagPass>();
  return v;
}

template <class R, int MODE>
int launch_mag(const PassCfg& pc, MagArgs<R> a, cudaStream_t s) {
  auto kern = k_mag_pass<R, MODE>;
  static std::atomic<uint64_t> configured{0};  // devices on which the attribute is set
  {
    const int rc_ = allow_smem_once(configured, (const void*)kern, (int)kSmemCap);
    if (rc_ != MMX_OK) return rc_;
  }
  a.outer = pc.outer;
  a.inner = pc.inner;
  a.P = pc.P;
  a.sP = pc.sP;
  kern<<<(unsigned)pc.tiles, pc.threads, pc.smem, s>>>(a);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

template <class R>
int dispatch_mag(const MagPass& mp, const MagArgs<R>& a, cudaStream_t s) {
  switch (mp.mode) {
    case MAG_E_FWD: return launch_mag<R, MAG_E_FWD>(mp.pc, a, s);
    case MAG_MID_FWD3: return launch_mag<R, MAG_MID_FWD3>(mp.pc, a, s);
    case MAG_MID_INV3: return launch_mag<R, MAG_MID_INV3>(mp.pc, a, s);
    case MAG_MID_FWD6: return launch_mag<R, MAG_MID_FWD6>(mp.pc, a, s);
    case MAG_MID_INV6: return launch_mag<R, MAG_MID_INV6>(mp.pc, a, s);
    case MAG_K_CURL_E: return launch_mag<R, MAG_K_CURL_E>(mp.pc, a, s);
    case MAG_K_GREEN: return launch_mag<R, MAG_K_GREEN>(mp.pc, a, s);
    case MAG_K_CURL: return launch_mag<R, MAG_K_CURL>(mp.pc, a, s);
    case MAG_MIX1: return launch_mag<R, MAG_MIX1>(mp.pc, a, s);
    case MAG_MIX2: return launch_mag<R, MAG_MIX2>(mp.pc, a, s);
    case MAG_UPDATE: return launch_mag<R, MAG_UPDATE>(mp.pc, a, s);
    default: return fail(MMX_ERR_ARG, "internal: unknown magnetic pass");
  }
}

// niter iterations on the fused schedule; work[0..4] hold A, B, U2, FFT(E) and the second field buffer.  The field
// is settled back into b->E (and cur to 0) at the end of the chunk.
template <class R>
int run_magnetic_fused(mmx_plan* p, const std::vector<MagPass>& passes, const mmx_magnetic_buffers* b,
                       mmx_rhs_state* st, int niter, cudaStream_t s) {
  using C = cpx<R>;
  MagArgs<R> a;
  memset(&a, 0, sizeof(a));
  a.N = p->N;
  a.ndim = p->ndim;
  for (int i = 0; i < 3; ++i) {
    a.dims[i] = (int)p->shape[i];
    a.kv[i] = p->kv_dev ? (const R*)p->kv_dev + p->kv_off[i] : nullptr;
  }
  a.inv_total = (R)(1.0 / (double)p->N);
  a.E0 = (C*)b->E;
  a.E1 = (C*)b->work[4];
  a.src = (const C*)b->src;
  a.ee = (const C*)b->chi_ee;
  a.eh = (const C*)b->chi_eh;
  a.he = (const C*)b->chi_he;
  a.hh = (const C*)b->chi_hh;
  a.A = (C*)b->work[0];
  a.B = (C*)b->work[1];
  a.U2 = (C*)b->work[2];
  a.Eh = (C*)b->work[3];
  a.st = st;
  a.partials = p->partials;
  a.done = p->done;
  for (int it = 0; it < niter; ++it) {
    for (const MagPass& mp : passes) {
      a.ax = p->ax[mp.axis];
      const int rc = dispatch_mag<R>(mp, a, s);
      if (rc != MMX_OK) return rc;
    }
  }
  const int64_t n3 = 3 * p->N;
  k_mag_settle<R><<<grid_blocks(n3, 256), 256, 0, s>>>(a.E0, a.E1, st, n3);
  k_mag_settle_state<<<1, 32, 0, s>>>(st);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

// niter iterations of the magnetic split-Richardson iteration with the decisions on the device (mmx_magnetic.cuh)
template <class R>
int run_magnetic(mmx_plan* p, const mmx_magnetic_buffers* b, mmx_rhs_state* st, int niter, cudaStream_t s) {
  using C = cpx<R>;
  const int64_t N = p->N, n3 = 3 * N;
  const KGrid g = kgrid_of(p);
  const R *k0 = kv_of<R>(p, 0), *k1 = kv_of<R>(p, 1), *k2 = kv_of<R>(p, 2);
  C* E = (C*)b->E;
  const C* src = (const C*)b->src;
  const C *ee = (const C*)b->chi_ee, *eh = (const C*)b->chi_eh, *he = (const C*)b->chi_he, *hh = (const C*)b->chi_hh;
  C *t = (C*)b->work[0], *u = (C*)b->work[1], *w = (C*)b->work[2], *dx = (C*)b->work[3], *d = (C*)b->work[4];
  C *F = (C*)b->work[5], *Eh = (C*)b->work[6];
  const int bv = grid_blocks(N, 256), b3 = grid_blocks(n3, 256);
  const int nb = (int)std::min<int64_t>(b3, p->partials_len / 3);
  const C zero = mkc<R>((R)0, (R)0);
  // One iteration with D = IFFT(i k x FFT(.)), in eight transforms instead of the reference's ten: the Green
  // function's input chi E + s' = u + D w + s' is transformed as FFT(u + s') + i k x FFT(w), and the curl of
  // t = G(...) - E is taken from the Green function's output minus FFT(E), both already in k-space.
  auto fft = [&](const C* in, C* out, int inv) { return run_fftn<R>(p, in, out, 3, inv, s); };
  auto curlk = [&](const C* Fin, C* out, const C* add, const C* sub) {
    k_curl_ft<R><<<bv, 256, 0, s>>>(Fin, out, g, k0, k1, k2, add, sub);
  };
  auto mix = [&](const C* x, const C* dxx) {
    k_chi_mix<R><<<bv, 256, 0, s>>>(x, dxx, ee, eh, he, hh, zero, zero, zero, zero, zero, u, w, N, st);
  };
  for (int it = 0; it < niter; ++it) {
    int rc;
    if ((rc = fft(E, Eh, 0)) != MMX_OK) return rc;           // Eh = FFT(E), kept
    curlk(Eh, F, nullptr, nullptr);
    if ((rc = fft(F, dx, 1)) != MMX_OK) return rc;           // dx = D E
    mix(E, dx);                                              // u = chi_EE E + chi_HE D E, w = chi_EH E + chi_HH D E
    if ((rc = fft(w, F, 0)) != MMX_OK) return rc;            // F = FFT(w)
    k_mag_usrc<R><<<b3, 256, 0, s>>>(t, u, src, st, n3);     // t = u + s'(alpha)
    if ((rc = fft(t, d, 0)) != MMX_OK) return rc;
    curlk(F, d, d, nullptr);                                 // d = FFT(u + s') + i k x FFT(w) = FFT(chi E + s')
    k_green_ft<R><<<bv, 256, 0, s>>>(d, g, k0, k1, k2, (R)0, (R)1, st);
    if ((rc = fft(d, t, 1)) != MMX_OK) return rc;
    k_axpby<R><<<b3, 256, 0, s>>>(t, t, E, mkc<R>((R)1, (R)0), mkc<R>((R)-1, (R)0), n3);  // t = G(...) - E
    curlk(d, F, nullptr, Eh);                                // F = i k x (FFT(t)), FFT(t) = G(...)^ - Eh
    if ((rc = fft(F, dx, 1)) != MMX_OK) return rc;           // dx = D t
    mix(t, dx);
    if ((rc = fft(w, F, 0)) != MMX_OK) return rc;
    curlk(F, d, nullptr, nullptr);
    if ((rc = fft(d, dx, 1)) != MMX_OK) return rc;           // dx = D w
    k_mag_update<R><<<nb, 256, 0, s>>>(d, u, dx, E, n3, p->partials);
    k_mag_decide<<<1, 256, 0, s>>>(p->partials, nb, st);
    k_mag_accept<R><<<b3, 256, 0, s>>>(E, d, st, n3);
    MMX_CUDA(cudaGetLastError());
  }
  return MMX_OK;
}
}  // namespace

extern "C" int mmx_magnetic_iterate(mmx_plan* p, const mmx_magnetic_buffers* b, mmx_rhs_state* st, int niter,
                                    int use_graph, void* stream) {
  if (!p || !b || !st || !b->E || !b->src || !b->chi_ee || !b->chi_eh || !b->chi_he || !b->chi_hh)
    return fail(MMX_ERR_ARG, "NULL plan or buffer");
  for (int i = 0; i < 7; ++i)
    if (!b->work[i]) return fail(MMX_ERR_ARG, "NULL work buffer");
  if (!p->kv_set) return fail(MMX_ERR_ARG, "k-vectors not set (mmx_plan_set_kvectors)");
  if (p->batch != 1 || p->ncomp != 1) return fail(MMX_ERR_ARG, "the plan must be a 1-component, 1-batch plan");
  if (niter < 1) return fail(MMX_ERR_ARG, "niter must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  // the composition of eight batched transforms (the faster one on the measured grids) unless MMX_MAG_FUSED=1 asks
  // for the fused pass schedule (2D and 3D grids)
  const char* fused_env = getenv("MMX_MAG_FUSED");
  const bool want_fused = fused_env && fused_env[0] == '1';
  const std::vector<MagPass> fused = want_fused ? build_mag_passes(p) : std::vector<MagPass>();
  auto run = [&](cudaStream_t cs) {
    if (!fused.empty())
      return p->prec == MMX_C128 ? run_magnetic_fused<double>(p, fused, b, st, niter, cs)
                                 : run_magnetic_fused<float>(p, fused, b, st, niter, cs);
    return p->prec == MMX_C128 ? run_magnetic<double>(p, b, st, niter, cs) : run_magnetic<float>(p, b, st, niter, cs);
  };
  if (!use_graph) return run(s);
  GraphKey key;
  key.ptrs = {(const void*)p, b->E, b->src, b->chi_ee, b->chi_eh, b->chi_he, b->chi_hh, (const void*)st};
  for (int i = 0; i < 7; ++i) key.ptrs.push_back(b->work[i]);
  key.ints = {fused.empty() ? -3 : -4, niter};  // a magnetic iteration chunk (-4: the fused schedule)
  cudaGraphExec_t exec = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_graph_mutex);
    for (const GraphEntry& ge : g_graphs)
      if (ge.key == key) exec = ge.exec;
  }
  if (!exec) {
    cudaStream_t cs = nullptr;
    MMX_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    int rc = e == cudaSuccess ? MMX_OK : cuda_fail(e, "cudaStreamBeginCapture");
    if (rc == MMX_OK) {
      rc = run(cs);
      e = cudaStreamEndCapture(cs, &graph);
      if (rc == MMX_OK && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamEndCapture");
    }
    if (rc == MMX_OK) {
      e = cudaGraphInstantiate(&exec, graph, 0);
      if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphInstantiate");
    }
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    if (rc != MMX_OK) return rc;
    std::lock_guard<std::mutex> lock(g_graph_mutex);
    g_graphs.push_back(GraphEntry{key, exec});
  }
  MMX_CUDA(cudaGraphLaunch(exec, s));
  return MMX_OK;
}

extern "C" int mmx_scalar_sigma(mmx_plan* p, const void* xp, int64_t nvox, double ab, double* out_dev, void* stream) {
  if (!p || !xp || !out_dev) return fail(MMX_ERR_ARG, "NULL plan or buffer");
  if (nvox < 1) return fail(MMX_ERR_ARG, "nvox must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  int blocks = grid_blocks(nvox, 256);
  if (2 * (int64_t)blocks > p->partials_len) blocks = (int)(p->partials_len / 2);
  k_scalar_sigma<<<blocks, 256, 0, s>>>((const double2*)xp, nvox, ab, p->partials);
  MMX_CUDA(cudaGetLastError());
  k_minmax_final<<<1, 256, 0, s>>>(p->partials, blocks, out_dev);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

extern "C" int mmx_chi_from_eps(const void* eps, int m, int64_t nvox, double s_re, double s_im, double d_re,
                                double d_im, void* chi, int precision, void* stream) {
  if (!eps || !chi) return fail(MMX_ERR_ARG, "NULL buffer");
  if (m != 1 && m != 9) return fail(MMX_ERR_ARG, "m must be 1 or 9");
  if (nvox < 1) return fail(MMX_ERR_ARG, "nvox must be positive");
  if (precision != MMX_C64 && precision != MMX_C128) return fail(MMX_ERR_ARG, "unknown precision");
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = grid_blocks((int64_t)m * nvox, 256);
  const double2 sc = make_double2(s_re, s_im), dc = make_double2(d_re, d_im);
  if (precision == MMX_C64)
    k_chi_from_eps<float2><<<blocks, 256, 0, s>>>((const double2*)eps, m, nvox, sc, dc, (float2*)chi);
  else
    k_chi_from_eps<double2><<<blocks, 256, 0, s>>>((const double2*)eps, m, nvox, sc, dc, (double2*)chi);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

// ---------------------------------------------------------------------------------------------------------------
// Allocation-free N-D FFT.
//
// The twiddle tables that a plan would allocate live in one file-scope device array instead, sized for three axes
// of at most MMX_NOALLOC_MAX_AXIS samples in complex128 (192 KiB, held by every GPU that loads this library until
// the process exits).  Each call rewrites the tables it needs for its own shape on its stream before the transform
// passes, so nothing has to start at zero; two calls that overlap on the GPU (different streams) overwrite each
// other's tables and race.  In host code the array's name is only a stand-in for the device symbol: the device
// address comes from cudaGetSymbolAddress, looked up once per device (on that device's first call).
// ---------------------------------------------------------------------------------------------------------------
#define MMX_NOALLOC_MAX_AXIS 4096

static __device__ __align__(256) unsigned char g_noalloc_twiddles[3 * MMX_NOALLOC_MAX_AXIS * sizeof(double2)];

namespace {

constexpr int kNoallocMaxDevices = 64;
void* g_noalloc_twiddle_ptr[kNoallocMaxDevices] = {};
std::mutex g_noalloc_mutex;

template <class R> __global__ void k_fill_twiddles(cpx<R>* __restrict__ tw, int n) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)t / (double)n, &s, &c);  // exp(-2 pi i t / n)
    tw[t] = mkc<R>((R)c, (R)s);
  }
}

int noalloc_scratch(void** out) {
  int dev = 0;
  MMX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocMaxDevices) return fail(MMX_ERR_UNSUPPORTED, "device ordinal too large");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_twiddle_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_twiddles);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_twiddles)");
    g_noalloc_twiddle_ptr[dev] = p;
  }
  *out = g_noalloc_twiddle_ptr[dev];
  return MMX_OK;
}

template <class R>
int fftn_noalloc(mmx_plan& desc, unsigned char* scratch, const void* in, void* out, int64_t nbatch, int inverse,
                 cudaStream_t s) {
  for (int i = 0; i < desc.ndim; ++i) {
    cpx<R>* tw = reinterpret_cast<cpx<R>*>(scratch + (size_t)i * MMX_NOALLOC_MAX_AXIS * sizeof(double2));
    const int n = (int)desc.shape[i];
    k_fill_twiddles<R><<<(n + 255) / 256, 256, 0, s>>>(tw, n);
    MMX_CUDA(cudaGetLastError());
    desc.ax[i].tw = tw;
  }
  return run_fftn<R>(&desc, in, out, nbatch, inverse, s);
}

}  // namespace

extern "C" int mmx_fftn_noalloc(int ndim, const int64_t* shape, const void* in, void* out, int64_t nbatch,
                                int inverse, int precision, void* stream) {
  if (ndim < 1 || ndim > 3) return fail(MMX_ERR_UNSUPPORTED, "grids of 1 to 3 axes are supported");
  if (!shape || !in || !out) return fail(MMX_ERR_ARG, "NULL shape or buffer");
  if (nbatch < 1) return fail(MMX_ERR_ARG, "nbatch must be positive");
  if (precision != MMX_C64 && precision != MMX_C128) return fail(MMX_ERR_ARG, "precision must be MMX_C64 or MMX_C128");
  mmx_plan desc;  // host-side descriptor only: no device memory is attached to it
  desc.ndim = ndim;
  desc.prec = precision;
  desc.N = 1;
  for (int i = 0; i < ndim; ++i) {
    if (shape[i] < 1 || shape[i] > MMX_NOALLOC_MAX_AXIS)
      return fail(MMX_ERR_UNSUPPORTED, "axis length " + std::to_string(shape[i]) +
                                           " exceeds the " + std::to_string(MMX_NOALLOC_MAX_AXIS) +
                                           "-sample limit of the allocation-free FFT (use mmx_fftn with a plan)");
    if (!factorize((int)shape[i], desc.ax[i]))
      return fail(MMX_ERR_UNSUPPORTED, "axis length " + std::to_string(shape[i]) +
                                           " has a prime factor above 13 (not supported)");
    desc.shape[i] = shape[i];
    desc.N *= shape[i];
  }
  void* scratch = nullptr;
  const int rc = noalloc_scratch(&scratch);
  if (rc != MMX_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (precision == MMX_C128) return fftn_noalloc<double>(desc, (unsigned char*)scratch, in, out, nbatch, inverse, s);
  return fftn_noalloc<float>(desc, (unsigned char*)scratch, in, out, nbatch, inverse, s);
}

// Scattering-matrix mode synthesis and detection (matrix.py:528-610, 685-755): scatter mode coefficients into rows of
// transverse spectra, or gather them back.
template <class R>
int mode_copy(bool scatter, const void* in, const int64_t* idx, int64_t nmodes, int64_t nrows, int64_t row_len,
              int conj, void* out, cudaStream_t s) {
  const int64_t total = nrows * nmodes;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>((total + threads - 1) / threads, (int64_t)sm_count() * 16);
  if (scatter)
    k_mode_scatter<R><<<(unsigned)blocks, threads, 0, s>>>((const cpx<R>*)in, idx, nmodes, nrows, row_len, conj,
                                                          (cpx<R>*)out);
  else
    k_mode_gather<R><<<(unsigned)blocks, threads, 0, s>>>((const cpx<R>*)in, idx, nmodes, nrows, row_len, conj,
                                                         (cpx<R>*)out);
  MMX_CUDA(cudaGetLastError());
  return MMX_OK;
}

int mode_args_ok(const void* in, const int64_t* idx, int64_t nmodes, int64_t nrows, int64_t row_len, void* out,
                 int precision) {
  if (!in || !idx || !out) return fail(MMX_ERR_ARG, "NULL buffer or mode table");
  if (nmodes < 0 || nrows < 0 || row_len < 1) return fail(MMX_ERR_ARG, "negative count or empty row");
  if (precision != MMX_C64 && precision != MMX_C128) return fail(MMX_ERR_ARG, "precision must be MMX_C64 or MMX_C128");
  return MMX_OK;
}

extern "C" int mmx_mode_scatter(const void* coef, const int64_t* idx, int64_t nmodes, int64_t nrows, int64_t row_len,
                                int conj, void* out, int precision, void* stream) {
  const int rc = mode_args_ok(coef, idx, nmodes, nrows, row_len, out, precision);
  if (rc != MMX_OK || nmodes == 0 || nrows == 0) return rc;
  if (precision == MMX_C128) return mode_copy<double>(true, coef, idx, nmodes, nrows, row_len, conj, out, (cudaStream_t)stream);
  return mode_copy<float>(true, coef, idx, nmodes, nrows, row_len, conj, out, (cudaStream_t)stream);
}

extern "C" int mmx_mode_gather(const void* in, const int64_t* idx, int64_t nmodes, int64_t nrows, int64_t row_len,
                               int conj, void* out, int precision, void* stream) {
  const int rc = mode_args_ok(in, idx, nmodes, nrows, row_len, out, precision);
  if (rc != MMX_OK || nmodes == 0 || nrows == 0) return rc;
  if (precision == MMX_C128) return mode_copy<double>(false, in, idx, nmodes, nrows, row_len, conj, out, (cudaStream_t)stream);
  return mode_copy<float>(false, in, idx, nmodes, nrows, row_len, conj, out, (cudaStream_t)stream);
}
