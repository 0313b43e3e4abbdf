// Host side of the fused iteration engine behind sp_engine_run (replaces
// phasing.iterate, phasing.py:181-289, for many trials at once).
//
// Trials are split into groups whose working set (psi, G and, for DM, G2)
// fits an L2 budget; each group runs its whole schedule before the next one
// starts, so its planes stay resident in the 126 MB L2 across iterations.
// Within a group, trials of the same size share one work list and each tick
// launches one column-pass and one row-pass kernel per size present.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include "sp_coherence.cuh"
#include "sp_common.cuh"
#include "sp_engine_launch.cuh"

namespace sp {

static cudaError_t launch_pass(int N, int E, int which, int grid, cudaStream_t st,
                               const PassArgs& a) {
  switch (N) {
    case 8: return launch_pass_n8(E, which, grid, st, a);
    case 16: return launch_pass_n16(E, which, grid, st, a);
    case 32: return launch_pass_n32(E, which, grid, st, a);
    case 64: return launch_pass_n64(E, which, grid, st, a);
    case 128: return launch_pass_n128(E, which, grid, st, a);
    case 256: return launch_pass_n256(E, which, grid, st, a);
    case 512: return launch_pass_n512(E, which, grid, st, a);
    case 1024: return launch_pass_n1024(E, which, grid, st, a);
    case 2048: return launch_pass_n2048(E, which, grid, st, a);
    case 4096: return launch_pass_n4096(E, which, grid, st, a);
    default: return cudaErrorInvalidValue;
  }
}

static cudaError_t pass_setup(int N, int E, int* occ) {
  switch (N) {
    case 8: return pass_setup_n8(E, occ);
    case 16: return pass_setup_n16(E, occ);
    case 32: return pass_setup_n32(E, occ);
    case 64: return pass_setup_n64(E, occ);
    case 128: return pass_setup_n128(E, occ);
    case 256: return pass_setup_n256(E, occ);
    case 512: return pass_setup_n512(E, occ);
    case 1024: return pass_setup_n1024(E, occ);
    case 2048: return pass_setup_n2048(E, occ);
    case 4096: return pass_setup_n4096(E, occ);
    default: return cudaErrorInvalidValue;
  }
}

static cudaError_t launch_pc(int N, int which, int grid, cudaStream_t st, const PcArgs& a) {
  switch (N) {
    case 8: return launch_pc_n8(which, grid, st, a);
    case 16: return launch_pc_n16(which, grid, st, a);
    case 32: return launch_pc_n32(which, grid, st, a);
    case 64: return launch_pc_n64(which, grid, st, a);
    case 128: return launch_pc_n128(which, grid, st, a);
    case 256: return launch_pc_n256(which, grid, st, a);
    case 512: return launch_pc_n512(which, grid, st, a);
    case 1024: return launch_pc_n1024(which, grid, st, a);
    case 2048: return launch_pc_n2048(which, grid, st, a);
    case 4096: return launch_pc_n4096(which, grid, st, a);
    default: return cudaErrorInvalidValue;
  }
}

static cudaError_t pc_setup_size(int N) {
  switch (N) {
    case 8: return pc_setup_n8();
    case 16: return pc_setup_n16();
    case 32: return pc_setup_n32();
    case 64: return pc_setup_n64();
    case 128: return pc_setup_n128();
    case 256: return pc_setup_n256();
    case 512: return pc_setup_n512();
    case 1024: return pc_setup_n1024();
    case 2048: return pc_setup_n2048();
    case 4096: return pc_setup_n4096();
    default: return cudaErrorInvalidValue;
  }
}

// Per device, per (logN, E): dynamic-smem attributes set and the resident CTAs
// per SM of the column pass ([0]) and row pass ([1]) cached.
static std::mutex g_setup_mutex;
static int g_occ[64][13][3][2];  // [device][log2 N][E = 8, 16, 32][pass]; 0 = not yet configured
static int g_sms[64];

static cudaError_t occupancy_for(int N, int E, int* occ, int* sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  const int l = ilog2(N), k = (E >= 32 ? 2 : (E >= 16 ? 1 : 0));
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_sms[dev] == 0) {
    e = cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
  }
  if (g_occ[dev][l][k][0] == 0) {
    int o[2] = {0, 0};
    e = pass_setup(N, E, o);
    if (e != cudaSuccess) return e;
    g_occ[dev][l][k][0] = std::max(1, o[0]);
    g_occ[dev][l][k][1] = std::max(1, o[1]);
  }
  occ[0] = g_occ[dev][l][k][0];
  occ[1] = g_occ[dev][l][k][1];
  *sms = g_sms[dev];
  return cudaSuccess;
}

// Per device, per logN: the partial-coherence kernels' dynamic-smem attribute.
static bool g_pc_ready[64][13];
static cudaError_t pc_ready(int N) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_pc_ready[dev][ilog2(N)]) {
    e = pc_setup_size(N);
    if (e != cudaSuccess) return e;
    g_pc_ready[dev][ilog2(N)] = true;
  }
  return cudaSuccess;
}

constexpr size_t kAlign = 256;
constexpr int kMinE = 8;  // smallest values-per-thread choice (most work items)
static inline size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

static bool uses_dm(const sp_trial& t) {
  for (int r = 0; r < t.n_runs; ++r)
    if (t.run_alg[r] == SP_DM && t.run_count[r] > 0) return true;
  return false;
}

// Does the trial project with a partially coherent divisor (ipsf and/or spectrum)?
static bool partial(const sp_trial& t) { return t.ipsf_dev != nullptr || t.spectrum_n > 0; }

static int default_e(int N) { return N >= 32 ? 32 : N; }

static int chosen_e(int N, const sp_run_opts* opts) {
  int E = default_e(N);
  if (opts) {
    const int l = ilog2(N);
    if (opts->e_per_logn[l] > 0) E = opts->e_per_logn[l];
  }
  return effective_e(N, E);
}

static int validate(const sp_trial& t, int idx) {
  SP_CHECK(is_pow2(t.n) && t.n >= kMinN && t.n <= kMaxN, SP_ERR_SIZE,
           "trial %d: N=%d must be a power of two in [%d, %d]", idx, t.n, kMinN, kMaxN);
  SP_CHECK(t.n_iter >= 0, SP_ERR_INVALID, "trial %d: n_iter < 0", idx);
  SP_CHECK(t.n_runs >= 1 && t.n_runs <= SP_MAX_RUNS, SP_ERR_INVALID,
           "trial %d: n_runs=%d not in [1, %d]", idx, t.n_runs, SP_MAX_RUNS);
  int period = 0;
  for (int r = 0; r < t.n_runs; ++r) {
    SP_CHECK(t.run_alg[r] >= SP_HIO && t.run_alg[r] <= SP_SF_CPU, SP_ERR_INVALID,
             "trial %d: unknown algorithm code %d", idx, t.run_alg[r]);
    SP_CHECK(t.run_count[r] >= 0, SP_ERR_INVALID, "trial %d: negative run count", idx);
    period += t.run_count[r];
  }
  SP_CHECK(period > 0, SP_ERR_INVALID, "trial %d: empty iteration order", idx);
  SP_CHECK(t.psi_dev && t.modulus_dev && t.support_dev, SP_ERR_INVALID,
           "trial %d: psi, modulus and support pointers are required", idx);
  SP_CHECK(((uintptr_t)t.psi_dev | (uintptr_t)t.modulus_dev | (uintptr_t)t.support_dev |
            (uintptr_t)t.ipsf_dev) % 16 == 0,
           SP_ERR_INVALID, "trial %d: psi, modulus, support and ipsf must be 16-byte aligned", idx);
  SP_CHECK(t.init == SP_INIT_GIVEN || t.init == SP_INIT_RANDOM_PHASE, SP_ERR_INVALID,
           "trial %d: unknown init mode %d", idx, t.init);
  SP_CHECK(t.spectrum_n >= 0 && t.spectrum_n <= 65536, SP_ERR_INVALID,
           "trial %d: spectrum_n=%d", idx, t.spectrum_n);
  SP_CHECK(t.spectrum_n == 0 || (t.spectrum_rescale_dev && t.spectrum_weight_dev), SP_ERR_INVALID,
           "trial %d: spectrum pointers are required when spectrum_n > 0", idx);
  if (uses_dm(t)) SP_CHECK(t.beta != 0.f, SP_ERR_INVALID, "trial %d: DM needs beta != 0", idx);
  if (t.save_dev) {
    SP_CHECK(t.r0 >= 0 && t.c0 >= 0 && t.rows > 0 && t.cols > 0 && t.r0 + t.rows <= t.n &&
                 t.c0 + t.cols <= t.n,
             SP_ERR_INVALID, "trial %d: crop box (%d,%d,%d,%d) outside %dx%d", idx, t.r0, t.c0,
             t.rows, t.cols, t.n, t.n);
  }
  return SP_OK;
}

struct Layout {
  size_t slots_off, items_off, planes_off, total;
  std::vector<size_t> g_off, g2_off;
  std::vector<size_t> mt_off;  // transposed modulus of each trial (shared by equal moduli)
  std::vector<int> mt_first;   // trials that own a transposed modulus (first use)
  std::vector<size_t> w_off, w2_off;  // partial-coherence divisor planes (0 = none)
  std::vector<size_t> p_off, p2_off;  // squared-divisor planes of spectrum trials (0 = none)
  size_t jobs_off;             // (slot, plane) jobs of the partial-coherence kernels
  int n_items, n_jobs;
};

static Layout layout_for(const sp_trial* trials, int n, const sp_run_opts* opts) {
  Layout L;
  L.slots_off = 0;
  L.items_off = align_up(sizeof(Slot) * (size_t)n);
  // reserve item slots for the smallest E (most items), so the size does not
  // depend on the radix choice
  (void)opts;
  int items = 0;
  for (int i = 0; i < n; ++i) {
    const int N = trials[i].n;
    items += N / lines_per_item(N, effective_e(N, kMinE));
  }
  L.n_items = items;
  int jobs = 0;
  for (int i = 0; i < n; ++i)
    if (partial(trials[i])) jobs += uses_dm(trials[i]) ? 2 : 1;
  L.n_jobs = jobs;
  L.jobs_off = L.items_off + align_up(sizeof(Item) * (size_t)std::max(items, 1));
  L.planes_off = L.jobs_off + align_up(sizeof(int2) * (size_t)std::max(jobs, 1));
  size_t off = L.planes_off;
  L.g_off.resize(n);
  L.g2_off.resize(n);
  for (int i = 0; i < n; ++i) {
    const size_t plane = (size_t)trials[i].n * trials[i].n * sizeof(float2);
    L.g_off[i] = off;
    off += align_up(plane);
    L.g2_off[i] = 0;
    if (uses_dm(trials[i])) {
      L.g2_off[i] = off;
      off += align_up(plane);
    }
  }
  // divisor planes of partially coherent trials, one per projection plane
  L.w_off.assign(n, 0);
  L.w2_off.assign(n, 0);
  L.p_off.assign(n, 0);
  L.p2_off.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    if (!partial(trials[i])) continue;
    const size_t px = (size_t)trials[i].n * trials[i].n;
    const bool dm = uses_dm(trials[i]), spec = trials[i].spectrum_n > 0;
    L.w_off[i] = off;
    off += align_up(px * sizeof(float2));
    if (dm) {
      L.w2_off[i] = off;
      off += align_up(px * sizeof(float2));
    }
    if (spec) {
      L.p_off[i] = off;
      off += align_up(px * sizeof(float));
      if (dm) {
        L.p2_off[i] = off;
        off += align_up(px * sizeof(float));
      }
    }
  }
  // one transposed copy per distinct (modulus, N), for the column pass
  std::map<std::pair<const float*, int>, size_t> seen;
  L.mt_off.resize(n);
  for (int i = 0; i < n; ++i) {
    const auto key = std::make_pair(trials[i].modulus_dev, trials[i].n);
    auto f = seen.find(key);
    if (f != seen.end()) {
      L.mt_off[i] = f->second;
      continue;
    }
    L.mt_off[i] = off;
    seen[key] = off;
    L.mt_first.push_back(i);
    off += align_up((size_t)trials[i].n * trials[i].n * sizeof(float));
  }
  L.total = off;
  return L;
}

// dst = src^T for an N x N float array (32 x 32 tiles through shared memory)
__global__ void transpose_kernel(const float* __restrict__ src, float* __restrict__ dst, int N) {
  __shared__ float tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y)
    tile[y][threadIdx.x] = src[(size_t)(by + y) * N + bx + threadIdx.x];
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y)
    dst[(size_t)(bx + y) * N + by + threadIdx.x] = tile[threadIdx.x][y];
}

// N = 8, 16: one block of N x N threads
__global__ void transpose_small_kernel(const float* __restrict__ src, float* __restrict__ dst, int N) {
  const int r = threadIdx.x / N, c = threadIdx.x % N;
  dst[c * N + r] = src[r * N + c];
}

static cudaError_t launch_transpose(const float* src, float* dst, int N, cudaStream_t st) {
  if (N >= 32)
    transpose_kernel<<<dim3(N / 32, N / 32), dim3(32, 8), 0, st>>>(src, dst, N);
  else
    transpose_small_kernel<<<1, N * N, 0, st>>>(src, dst, N);
  return cudaGetLastError();
}

// one launch target: the items of one size within one group
struct Segment {
  int N, E, first, count, grid[2];  // grid[pass]: 0 column, 1 row
  int pc_first, pc_count, pc_grid;  // partial-coherence jobs of this size
  int pc_egrid;                     // grid of the tiled rescale kernel
  int col_ticks;                    // the column pass runs at ticks [0, col_ticks)
  int pc_mask;                      // partial-coherence kernels launched (bit = which)
  int ticks;                        // ticks of this segment's longest trial (n_iter + 1)
};

struct GraphKey {
  void* ws;
  int dev, group, n_ticks;
  std::vector<int> shape;  // flattened segments
  bool operator<(const GraphKey& o) const {
    return std::tie(ws, dev, group, n_ticks, shape) <
           std::tie(o.ws, o.dev, o.group, o.n_ticks, o.shape);
  }
};
static std::mutex g_graph_mutex;
static std::map<GraphKey, cudaGraphExec_t> g_graphs;
static thread_local int64_t g_last_launches = 0;

// One segment's launch chain: per tick its partial-coherence kernels, its
// column pass and its row pass.
static int launch_segment(const Segment& sg, const Slot* slots, const Item* items,
                          const int2* jobs, const float2* tw, cudaStream_t st) {
  for (int k = 0; k < sg.ticks; ++k) {
    // partially coherent projections first (their slots sit out the column pass)
    if (sg.pc_count > 0) {
      PcArgs pa{slots, jobs + sg.pc_first, sg.pc_count, k, tw};
      for (int which = 0; which < 5; ++which)
        if (sg.pc_mask & (1 << which))
          SP_CUDA_TRY(launch_pc(sg.N, which, which == 3 ? sg.pc_egrid : sg.pc_grid, st, pa));
    }
    for (int which = 0; which < 2; ++which) {
      if (which == 0 && k >= sg.col_ticks) continue;  // no column work left in this segment
      // the column pass walks the items backwards: it starts on the trials
      // whose G planes the row pass wrote last (still in L2), and the next
      // row pass starts on the ones it wrote last
      PassArgs a{slots, items + sg.first, sg.count, nullptr, k, tw, which == 0 ? 1 : 0};
      SP_CUDA_TRY(launch_pass(sg.N, sg.E, which, sg.grid[which], st, a));
    }
  }
  return SP_OK;
}

// Auxiliary streams and events of the calling thread, per device, for the
// concurrent segment chains (created before any capture begins), released
// when the thread exits (errors ignored: at process exit the runtime may
// already be shutting down).
struct ForkPool {
  int dev = -1;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;  // [0] fork, [1 + i] join of stream i
  ForkPool() = default;
  ForkPool(const ForkPool&) = delete;
  ForkPool& operator=(const ForkPool&) = delete;
  ~ForkPool() {
    if (dev < 0 || (streams.empty() && events.empty()) || cudaSetDevice(dev) != cudaSuccess) return;
    for (cudaStream_t s : streams) cudaStreamDestroy(s);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
  }
};
static thread_local std::map<int, ForkPool> t_fork;

static cudaError_t fork_pool(int dev, int branches, ForkPool** out) {
  ForkPool& P = t_fork[dev];
  P.dev = dev;
  while ((int)P.streams.size() < branches) {
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    P.streams.push_back(s);
  }
  while ((int)P.events.size() < branches + 1) {
    cudaEvent_t ev = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
    P.events.push_back(ev);
  }
  *out = &P;
  return cudaSuccess;
}

// Every segment of a group, each as its own chain: segments share no data
// (their trials, planes and items are disjoint; slots, items and transposed
// moduli are only read), so the chains of different sizes run concurrently
// -- the first on `st`, the others on auxiliary streams forked from it and
// joined back into it (in a capture this forms parallel graph branches).  The
// joins are made even after a failed launch, so a capture never ends with
// unjoined work.
static int launch_ticks(const std::vector<Segment>& segs, const Slot* slots, const Item* items,
                        const int2* jobs, const float2* tw, ForkPool* P, cudaStream_t st) {
  if (segs.size() == 1 || P == nullptr) {
    for (const Segment& sg : segs) {
      const int rc = launch_segment(sg, slots, items, jobs, tw, st);
      if (rc != SP_OK) return rc;
    }
    return SP_OK;
  }
  const int n_aux = (int)segs.size() - 1;
  SP_CUDA_TRY(cudaEventRecord(P->events[0], st));
  int rc = SP_OK;
  int forked = 0;
  for (int i = 0; i < n_aux; ++i) {
    if (cudaStreamWaitEvent(P->streams[i], P->events[0], 0) != cudaSuccess) {
      set_error("cudaStreamWaitEvent failed while forking segment %d", i + 1);
      rc = SP_ERR_CUDA;
      break;
    }
    forked = i + 1;
    if (rc == SP_OK) rc = launch_segment(segs[i + 1], slots, items, jobs, tw, P->streams[i]);
  }
  if (rc == SP_OK) rc = launch_segment(segs[0], slots, items, jobs, tw, st);
  for (int i = 0; i < forked; ++i) {
    const cudaError_t e1 = cudaEventRecord(P->events[1 + i], P->streams[i]);
    const cudaError_t e2 = cudaStreamWaitEvent(st, P->events[1 + i], 0);
    if (rc == SP_OK && (e1 != cudaSuccess || e2 != cudaSuccess)) {
      set_error("joining segment %d failed: %s", i + 1,
                cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
      rc = SP_ERR_CUDA;
    }
  }
  return rc;
}

}  // namespace sp

using namespace sp;

extern "C" int sp_engine_workspace_size(const sp_trial* trials, int n_trials, size_t* bytes) {
  SP_CHECK(bytes != nullptr, SP_ERR_INVALID, "bytes is null");
  SP_CHECK(n_trials >= 0 && (n_trials == 0 || trials), SP_ERR_INVALID, "no trials");
  for (int i = 0; i < n_trials; ++i) {
    SP_CHECK(is_pow2(trials[i].n) && trials[i].n >= kMinN && trials[i].n <= kMaxN, SP_ERR_SIZE,
             "trial %d: N=%d must be a power of two in [%d, %d]", i, trials[i].n, kMinN, kMaxN);
  }
  *bytes = layout_for(trials, n_trials, nullptr).total;
  return SP_OK;
}

// sp_engine_run's body; `concurrent` lets the chains of different sizes run
// on forked auxiliary streams (sp_engine_run_static keeps them on `stream`:
// it creates no streams or events).
int sp::engine_run(const sp_trial* trials, int n_trials, void* workspace_dev, size_t workspace_bytes,
                   const sp_run_opts* opts, sp_stream_t stream, bool concurrent) {
  SP_CHECK(n_trials >= 0, SP_ERR_INVALID, "n_trials < 0");
  if (n_trials == 0) return SP_OK;
  SP_CHECK(trials != nullptr, SP_ERR_INVALID, "trials is null");
  for (int i = 0; i < n_trials; ++i) {
    const int st = validate(trials[i], i);
    if (st != SP_OK) return st;
  }
  const Layout L = layout_for(trials, n_trials, opts);
  SP_CHECK(workspace_dev != nullptr && workspace_bytes >= L.total, SP_ERR_WORKSPACE,
           "workspace of %zu bytes given, %zu needed", workspace_bytes, L.total);
  cudaStream_t st = as_stream(stream);
  const float2* tw = nullptr;
  SP_CUDA_TRY(twiddles(&tw));
  char* ws = static_cast<char*>(workspace_dev);
  int dev = 0;
  SP_CUDA_TRY(cudaGetDevice(&dev));

  // groups of consecutive trials whose working set fits the L2 budget
  const int64_t budget = opts ? opts->l2_group_bytes : 0;
  std::vector<int> gstart{0};
  int64_t acc = 0;
  for (int i = 0; i < n_trials; ++i) {
    const int64_t plane = (int64_t)trials[i].n * trials[i].n * 8;
    const int64_t need = plane * (uses_dm(trials[i]) ? 3 : 2);
    if (budget > 0 && i > gstart.back() && acc + need > budget) {
      gstart.push_back(i);
      acc = 0;
    }
    acc += need;
  }
  gstart.push_back(n_trials);
  const int n_groups = (int)gstart.size() - 1;

  // slot descriptors and, per group and size, a contiguous run of items
  std::vector<Slot> hs(n_trials);
  std::vector<Item> hi;
  hi.reserve(L.n_items);
  std::vector<int2> hj;  // partial-coherence jobs (slot, plane)
  hj.reserve(L.n_jobs);
  std::vector<std::vector<Segment>> segs(n_groups);
  std::vector<int> ticks(n_groups, 0);
  for (int g = 0; g < n_groups; ++g) {
    for (int N = kMinN; N <= kMaxN; N *= 2) {
      const int E = chosen_e(N, opts);
      const int L_items = N / lines_per_item(N, E);
      const int first = (int)hi.size();
      for (int i = gstart[g]; i < gstart[g + 1]; ++i) {
        if (trials[i].n != N) continue;
        for (int b = 0; b < L_items; ++b) hi.push_back(Item{i, b});
      }
      const int count = (int)hi.size() - first;
      if (count == 0) continue;
      int occ[2] = {1, 1}, sms = 1;
      SP_CUDA_TRY(occupancy_for(N, E, occ, &sms));
      Segment sg{N, E, first, count, {1, 1}, (int)hj.size(), 0, 1, 1, 0, 0, 0};
      for (int i = gstart[g]; i < gstart[g + 1]; ++i)
        if (trials[i].n == N) sg.ticks = std::max(sg.ticks, trials[i].n_iter + 1);
      // Partially coherent slots project in their own kernels: the column
      // pass has work for them only at tick 0, to start a random phase.  A
      // segment of such slots alone launches it only while it has work.
      for (int i = gstart[g]; i < gstart[g + 1]; ++i) {
        if (trials[i].n != N) continue;
        if (!partial(trials[i])) sg.col_ticks = INT32_MAX;
        else if (trials[i].init == SP_INIT_RANDOM_PHASE) sg.col_ticks = std::max(sg.col_ticks, 1);
      }
      for (int p = 0; p < 2; ++p) {
        int per_sm = occ[p];
        if (opts && opts->ctas_per_sm > 0) per_sm = std::min(per_sm, (int)opts->ctas_per_sm);
        const int units = p == 0 ? count * col_split(N, E) : count;
        sg.grid[p] = std::max(1, std::min(units, sms * per_sm));
      }
      for (int i = gstart[g]; i < gstart[g + 1]; ++i) {
        if (trials[i].n != N || !partial(trials[i])) continue;
        hj.push_back(int2{i, 0});
        if (uses_dm(trials[i])) hj.push_back(int2{i, 1});
      }
      sg.pc_count = (int)hj.size() - sg.pc_first;
      // A and B always; W with an ipsf; R with a spectrum; B1 with both
      for (int i = gstart[g]; i < gstart[g + 1]; ++i) {
        if (trials[i].n != N || !partial(trials[i])) continue;
        const bool ip = trials[i].ipsf_dev != nullptr, sp = trials[i].spectrum_n > 0;
        sg.pc_mask |= 1 | 16 | (ip ? 2 : 0) | (sp ? 8 : 0) | (ip && sp ? 4 : 0);
      }
      if (sg.pc_count > 0) {
        SP_CUDA_TRY(pc_ready(N));
        const int per_job = N / lines_per_item(N, pc_e(N));
        sg.pc_grid = std::max(1, std::min(sg.pc_count * per_job, sms * 4));
        const int64_t tiles = (int64_t)sg.pc_count * N * N / rescale_tile_pixels(N);
        sg.pc_egrid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sms * 8));
      }
      segs[g].push_back(sg);
    }
    for (int i = gstart[g]; i < gstart[g + 1]; ++i) {
      const sp_trial& t = trials[i];
      ticks[g] = std::max(ticks[g], t.n_iter + 1);
      Slot& s = hs[i];
      memset(&s, 0, sizeof(Slot));
      s.logn = ilog2(t.n);
      s.n_iter = t.n_iter;
      s.n_runs = t.n_runs;
      s.init = t.init;
      int end = 0;
      for (int r = 0; r < SP_MAX_RUNS; ++r) {
        if (r < t.n_runs) {
          end += t.run_count[r];
          s.run_alg[r] = t.run_alg[r];
        }
        s.run_end[r] = end;
      }
      s.beta = t.beta;
      s.seed = t.seed;
      s.trial = t.trial;
      s.r0 = t.r0;
      s.c0 = t.c0;
      s.rows = t.rows;
      s.cols = t.cols;
      s.start_tick = 0;
      s.psi = static_cast<float2*>(t.psi_dev);
      s.g = reinterpret_cast<float2*>(ws + L.g_off[i]);
      s.g2 = L.g2_off[i] ? reinterpret_cast<float2*>(ws + L.g2_off[i]) : nullptr;
      s.modulus = t.modulus_dev;
      s.modulus_t = reinterpret_cast<const float*>(ws + L.mt_off[i]);
      s.support = t.support_dev;
      s.save = static_cast<float2*>(t.save_dev);
      s.err = t.errors_dev;
      s.ipsf = static_cast<const float2*>(t.ipsf_dev);
      s.w = L.w_off[i] ? reinterpret_cast<float2*>(ws + L.w_off[i]) : nullptr;
      s.w2 = L.w2_off[i] ? reinterpret_cast<float2*>(ws + L.w2_off[i]) : nullptr;
      s.spec_n = t.spectrum_n;
      s.spec_r = t.spectrum_n ? t.spectrum_rescale_dev : nullptr;
      s.spec_w = t.spectrum_n ? t.spectrum_weight_dev : nullptr;
      s.p = L.p_off[i] ? reinterpret_cast<float*>(ws + L.p_off[i]) : nullptr;
      s.p2 = L.p2_off[i] ? reinterpret_cast<float*>(ws + L.p2_off[i]) : nullptr;
    }
  }
  SP_CHECK((int)hi.size() <= L.n_items, SP_ERR_INVALID,
           "internal: %zu work items exceed the %d reserved", hi.size(), L.n_items);
  SP_CHECK((int)hj.size() == L.n_jobs, SP_ERR_INVALID,
           "internal: %zu partial-coherence jobs, %d reserved", hj.size(), L.n_jobs);
  SP_CUDA_TRY(cudaMemcpyAsync(ws + L.slots_off, hs.data(), sizeof(Slot) * hs.size(),
                              cudaMemcpyHostToDevice, st));
  if (!hi.empty())
    SP_CUDA_TRY(cudaMemcpyAsync(ws + L.items_off, hi.data(), sizeof(Item) * hi.size(),
                                cudaMemcpyHostToDevice, st));
  if (!hj.empty())
    SP_CUDA_TRY(cudaMemcpyAsync(ws + L.jobs_off, hj.data(), sizeof(int2) * hj.size(),
                                cudaMemcpyHostToDevice, st));
  for (int i = 0; i < n_trials; ++i) {
    if (trials[i].errors_dev && trials[i].n_iter > 0)
      SP_CUDA_TRY(cudaMemsetAsync(trials[i].errors_dev, 0,
                                  sizeof(double) * 2 * (size_t)trials[i].n_iter, st));
  }
  // the column pass reads each modulus transposed (rows of the copy are columns)
  for (int i : L.mt_first)
    SP_CUDA_TRY(launch_transpose(trials[i].modulus_dev, reinterpret_cast<float*>(ws + L.mt_off[i]),
                                 trials[i].n, st));
  const Slot* dslots = reinterpret_cast<const Slot*>(ws + L.slots_off);
  const Item* ditems = reinterpret_cast<const Item*>(ws + L.items_off);
  const int2* djobs = reinterpret_cast<const int2*>(ws + L.jobs_off);
  const bool use_graph = opts && opts->use_graph && st != nullptr;
  g_last_launches = (int64_t)L.mt_first.size();
  size_t max_segs = 1;
  for (int g = 0; g < n_groups; ++g) {
    max_segs = std::max(max_segs, segs[g].size());
    for (const Segment& sg : segs[g]) {
      g_last_launches += sg.ticks + std::min(sg.ticks, sg.col_ticks);
      g_last_launches += (int64_t)__builtin_popcount(sg.pc_mask) * sg.ticks;
    }
  }
  // auxiliary streams for concurrent segment chains, made before any capture
  ForkPool* pool = nullptr;
  if (concurrent && max_segs > 1) SP_CUDA_TRY(fork_pool(dev, (int)max_segs - 1, &pool));

  for (int g = 0; g < n_groups; ++g) {
    if (!use_graph) {
      const int rc = launch_ticks(segs[g], dslots, ditems, djobs, tw, pool, st);
      if (rc != SP_OK) return rc;
      continue;
    }
    GraphKey key{workspace_dev, dev, g, ticks[g], {}};
    for (const Segment& sg : segs[g])
      key.shape.insert(key.shape.end(), {sg.N, sg.E, sg.first, sg.count, sg.grid[0], sg.grid[1],
                                         sg.pc_first, sg.pc_count, sg.pc_grid, sg.pc_egrid,
                                         std::min(sg.ticks, sg.col_ticks), sg.pc_mask, sg.ticks});
    cudaGraphExec_t exec = nullptr;
    {
      std::lock_guard<std::mutex> lock(g_graph_mutex);
      auto f = g_graphs.find(key);
      if (f != g_graphs.end()) exec = f->second;
    }
    if (!exec) {
      cudaGraph_t graph = nullptr;
      SP_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      const int rc = launch_ticks(segs[g], dslots, ditems, djobs, tw, pool, st);
      const cudaError_t ce = cudaStreamEndCapture(st, &graph);
      if (rc != SP_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      SP_CUDA_TRY(ce);
      const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      SP_CUDA_TRY(ie);
      std::lock_guard<std::mutex> lock(g_graph_mutex);
      g_graphs[key] = exec;
    }
    SP_CUDA_TRY(cudaGraphLaunch(exec, st));
  }
  return SP_OK;
}

extern "C" int sp_engine_run(const sp_trial* trials, int n_trials, void* workspace_dev,
                             size_t workspace_bytes, const sp_run_opts* opts, sp_stream_t stream) {
  return engine_run(trials, n_trials, workspace_dev, workspace_bytes, opts, stream, true);
}

extern "C" int64_t sp_engine_last_launches(void) { return g_last_launches; }

extern "C" int64_t sp_engine_graph_count(void) {
  std::lock_guard<std::mutex> lock(g_graph_mutex);
  return (int64_t)g_graphs.size();
}

extern "C" int sp_engine_release_device_graphs(void) {
  int dev = 0;
  SP_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_graph_mutex);
  for (auto it = g_graphs.begin(); it != g_graphs.end();) {
    if (it->first.dev == dev) {
      cudaGraphExecDestroy(it->second);
      it = g_graphs.erase(it);
    } else {
      ++it;
    }
  }
  return SP_OK;
}

extern "C" int sp_engine_release_graphs(void) {
  std::lock_guard<std::mutex> lock(g_graph_mutex);
  for (auto& kv : g_graphs) cudaGraphExecDestroy(kv.second);
  g_graphs.clear();
  return SP_OK;
}
