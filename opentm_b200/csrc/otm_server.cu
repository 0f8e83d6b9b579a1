// otm_server.cu -- serving of independent homogenization requests on one GPU, in two forms.
//
// Handle form (default): the server keeps a few streams ("lanes"). An admitted request runs on
// an idle lane as one resident solver handle (otm::Homo, the same object otm_homo_* drives):
// the field goes up from the lane's pinned staging buffer, update() builds the coarse
// operators, and the whole preconditioned-CG loop runs on the device as one conditional-graph
// launch, followed by the K^H reduction and a copy of the solve scalars to pinned memory and an
// event. Scheduling never waits for a lane except when the queue is blocked; lanes overlap on
// the GPU, so the small kernels of one request fill the gaps of another. Handles stay resident
// per lane and size after their request finishes and are reused by the next request of that
// size (a handle is built, and its solve graph captured, once); idle handles are destroyed,
// least recently used first, when a new one would not fit the memory budget.
//
// Batched form: each admitted request owns a resident multigrid hierarchy (an otm::Homo in
// server mode: the server's stream, buffers from the server's memory pool). Its device
// pointers are collected in a ReqDesc that lives in a device-side slot table; a batched launch
// carries a small task list (slot, level, first block, block count) and every block finds its
// task by binary search, then runs the same device body as the single-request kernel. One
// scheduling step advances all running requests by a few preconditioned-CG iterations: per
// multigrid level one launch per colour pass / residual / restriction / prolongation over every
// request that has that level, one launch of the single-CTA tails (one block per request) and
// one launch per Krylov update. Requests finish, release their memory and are replaced by
// queued ones at step boundaries.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include "opentm_b200_server.h"
#include "otm_homo_impl.h"
#include "otm_host_ring.h"

namespace otm {

constexpr int kSrvMaxLevels = 12;
constexpr int kSrvMaxActive = 256;
constexpr int kSrvMaxStreams = 64;

struct ReqLevel {
  Dims d;
  float* u;
  float* f;
  float* r;
  const float* st;
};

struct ReqDesc {
  int nlev, tail_l, nc, pad;
  ReqLevel lv[kSrvMaxLevels];
  const float* ks;
  float* x;
  float* p;
  float* q;
  double* partials;
  SolveScalars* sc;
  FineOp op;
  TailDesc tail;
};

struct BTask {
  int slot;
  int level;
  int blk0;
  int nblk;
};

struct SlotStatus {
  int done, nan, iter, pad;
  double relres[3];
  double kh[6];
};

__device__ __forceinline__ int find_task(const BTask* __restrict__ t, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&t[mid].blk0) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

#define OTM_TASK_PROLOGUE                                   \
  const int ti = find_task(tasks, n, int(blockIdx.x));      \
  const BTask T = tasks[ti];                                \
  const ReqDesc& D = R[T.slot];                             \
  if (solve_done(D.sc)) return;                             \
  const unsigned int lblk = blockIdx.x - unsigned(T.blk0);  \
  const size_t tid = size_t(lblk) * blockDim.x + threadIdx.x;

static __global__ void __launch_bounds__(kBlock) kb_zero(const BTask* __restrict__ tasks, int n,
                                                         const ReqDesc* __restrict__ R) {
  OTM_TASK_PROLOGUE
  const ReqLevel& L = D.lv[T.level];
  if (tid < 3 * L.d.nv()) L.u[tid] = 0.f;
}

static __global__ void __launch_bounds__(kBlock) kb_gs(const BTask* __restrict__ tasks, int n,
                                                       const ReqDesc* __restrict__ R, int color) {
  OTM_TASK_PROLOGUE
  const ReqLevel& L = D.lv[T.level];
  if (T.level == 0)  // colour pair on the fine level
    gs_fine_pair_body<3, float, float>(L.d, color, D.ks, D.op, L.u, L.f, nullptr, tid);
  else
    gs_coarse_body<3>(L.d, color, L.st, L.u, L.f, tid);
}

static __global__ void __launch_bounds__(kBlock) kb_resid(const BTask* __restrict__ tasks, int n,
                                                          const ReqDesc* __restrict__ R) {
  OTM_TASK_PROLOGUE
  const ReqLevel& L = D.lv[T.level];
  if (T.level == 0)
    resid_fine_body<false, 3, float, float>(L.d, D.ks, D.op, L.u, L.f, L.r, nullptr, tid);
  else
    resid_coarse_body<3>(L.d, L.st, L.u, L.f, L.r, tid);
}

static __global__ void __launch_bounds__(kBlock) kb_restrict(const BTask* __restrict__ tasks, int n,
                                                             const ReqDesc* __restrict__ R) {
  OTM_TASK_PROLOGUE
  const ReqLevel& L = D.lv[T.level];
  const ReqLevel& C = D.lv[T.level + 1];
  restrict_body<3, float>(L.d, C.d, L.r, C.f, tid);
}

static __global__ void __launch_bounds__(kBlock) kb_prolong(const BTask* __restrict__ tasks, int n,
                                                            const ReqDesc* __restrict__ R) {
  OTM_TASK_PROLOGUE
  const ReqLevel& L = D.lv[T.level];
  const ReqLevel& C = D.lv[T.level + 1];
  prolong_body<3, float>(L.d, C.d, C.u, L.u, tid);
}

static __global__ void __launch_bounds__(kTailThreads) kb_tail(const BTask* __restrict__ tasks, int n,
                                                               const ReqDesc* __restrict__ R) {
  const ReqDesc& D = R[tasks[blockIdx.x].slot];
  if (solve_done(D.sc)) return;
  extern __shared__ float sm[];
  vcycle_tail_body(D.tail, sm);
}

static __global__ void __launch_bounds__(kBlock) kb_dot_rz(const BTask* __restrict__ tasks, int n,
                                                           const ReqDesc* __restrict__ R) {
  OTM_TASK_PROLOGUE
  (void)tid;
  dot_rz_body(D.lv[0].d.nv(), D.lv[0].f, D.lv[0].u, D.partials, D.sc, lblk, unsigned(T.nblk));
}

static __global__ void __launch_bounds__(kBlock) kb_update_p(const BTask* __restrict__ tasks, int n,
                                                             const ReqDesc* __restrict__ R) {
  OTM_TASK_PROLOGUE
  update_p_body(D.lv[0].d.nv(), D.lv[0].u, D.p, D.sc, tid);
}

static __global__ void __launch_bounds__(kBlock) kb_apply_dot(const BTask* __restrict__ tasks, int n,
                                                              const ReqDesc* __restrict__ R) {
  OTM_TASK_PROLOGUE
  (void)tid;
  apply_dot_body<false>(D.lv[0].d, D.ks, D.op, D.p, D.q, D.partials, D.sc, lblk, unsigned(T.nblk));
}

static __global__ void __launch_bounds__(kBlock) kb_update_xr(const BTask* __restrict__ tasks, int n,
                                                              const ReqDesc* __restrict__ R, int max_iter) {
  OTM_TASK_PROLOGUE
  (void)tid;
  update_xr_body(D.lv[0].d.nv(), D.x, D.lv[0].f, D.p, D.q, D.partials, D.sc, max_iter, lblk, unsigned(T.nblk));
}

// Convergence state (and K^H once computed) of every listed slot in one array.
static __global__ void kb_gather(const int* __restrict__ slots, int n, const ReqDesc* __restrict__ R,
                                 SlotStatus* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SolveScalars* sc = R[slots[i]].sc;
  SlotStatus s;
  s.done = sc->done;
  s.nan = sc->nan;
  s.iter = sc->iter;
  s.pad = 0;
  for (int c = 0; c < 3; c++) s.relres[c] = sc->relres[c];
  for (int c = 0; c < 6; c++) s.kh[c] = sc->kh[c];
  out[i] = s;
}

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Pinned host memory for submitted fields (offsets kept by RingOffsets). A full ring leaves the
// field in pageable memory.
class HostRing {
 public:
  ~HostRing() {
    if (base_) cudaFreeHost(base_);
  }
  cudaError_t init(size_t bytes) {
    const size_t n = bytes / sizeof(float);
    if (n == 0) return cudaSuccess;
    const cudaError_t e = cudaMallocHost((void**)&base_, n * sizeof(float));
    if (e != cudaSuccess) {
      base_ = nullptr;
      return e;
    }
    off_ = RingOffsets(n, 64);  // 256-byte starts
    return cudaSuccess;
  }
  float* alloc(size_t n, int64_t* seq) {
    size_t o = 0;
    if (!base_ || !off_.alloc(n, &o, seq)) return nullptr;
    return base_ + o;
  }
  void release(int64_t seq) { off_.release(seq); }

 private:
  float* base_ = nullptr;
  RingOffsets off_;
};

struct Request {
  int64_t id = 0;
  int reso[3] = {0, 0, 0};
  std::vector<float> k;      // the field, when the pinned ring had no room
  float* pinned = nullptr;   // the field in the pinned ring
  int64_t ring_seq = -1;
  const float* field() const { return pinned ? pinned : k.data(); }
  int state = 0;  // 0 queued, 1 running, 2 done, 3 cancelled, 4 failed
  int status = OTM_ERR_NOT_READY;
  bool cancel = false;
  double C[9] = {};
  otm_request_info info{};
  size_t bytes = 0;
  int slot = -1;
  std::unique_ptr<Homo> h;
};

static void homo_config(const otm_server_config& sc, const int reso[3], otm_config* c) {
  otm_config_init(c);
  for (int i = 0; i < 3; i++) c->reso[i] = reso[i];
  c->fem_rel_thres = sc.fem_rel_thres;
  c->max_iter = sc.max_iter;
  c->pre_smooth = sc.pre_smooth;
  c->post_smooth = sc.pre_smooth;
  c->solver = OTM_SOLVER_PCG;
  c->precision = OTM_PRECISION_FP32;
  c->power_penal = sc.power_penal;
  c->use_graphs = 0;
}

// Device bytes of one request's resident state (the allocations of Homo::build for an FP32
// PCG solve).
static size_t request_bytes(const int reso[3]) {
  size_t total = 0;
  Dims d{reso[0], reso[1], reso[2]};
  int L = 0;
  while (true) {
    const size_t nv = d.nv();
    total += 9 * nv * sizeof(float);  // u, f, r
    if (L > 0) total += 27 * nv * sizeof(float);
    L++;
    const bool can = d.nx % 2 == 0 && d.ny % 2 == 0 && d.nz % 2 == 0 && d.nx >= 8 && d.ny >= 8 && d.nz >= 8 &&
                     nv > 64;
    if (!can) break;
    d = Dims{d.nx / 2, d.ny / 2, d.nz / 2};
  }
  const size_t nv0 = size_t(reso[0]) * reso[1] * reso[2];
  const size_t nc = d.nv();
  total += nv0 * sizeof(float) * (2 + 4 * 3);  // ks, kraw, b, x, p, q
  total += nc * nc * sizeof(double) + 64 * 27 * sizeof(float);
  total += sizeof(SolveScalars) + size_t(kMaxPartials) * 16 * sizeof(double) + 8 * sizeof(double) + 16;
  total += nv0 * sizeof(float);  // the imported field while it is being set up
  return total;
}

}  // namespace otm

using namespace otm;

namespace otm {

// A resident handle of one cell size on a lane.
struct CachedHandle {
  int reso[3] = {0, 0, 0};
  std::unique_ptr<Homo> h;
  size_t bytes = 0;
  uint64_t last_use = 0;
};

// One stream of the handle form: at most one running request, handles kept per cell size.
struct Lane {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;  // recorded after the running request's last copy
  int64_t req = -1;            // running request (-1: idle)
  Homo* run = nullptr;         // its handle
  std::vector<CachedHandle> cache;
  float* stage = nullptr;  // pinned copy of the running request's field
  size_t stage_cap = 0;    // floats
};

}  // namespace otm

struct otm_server {
  otm_server_config cfg{};
  bool handles = false;  // handle form
  std::vector<otm::Lane> lanes;
  size_t bytes_resident = 0;  // all handles of the handle form, running or idle
  uint64_t use_clock = 0;
  otm::HostRing ring;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  std::map<int64_t, Request> reqs;
  std::deque<int64_t> queue;
  std::vector<int64_t> slots;  // request id per slot (-1 free)
  size_t bytes_in_use = 0;
  int64_t next_id = 1;
  ReqDesc* d_desc = nullptr;
  BTask* d_tasks = nullptr;
  size_t task_cap = 0;
  int* d_slots = nullptr;
  SlotStatus* d_status = nullptr;
  SlotStatus* h_status = nullptr;
  // pinned staging of the admitted requests' fields; reused once its copies are done
  float* h_stage = nullptr;
  size_t stage_cap = 0, stage_used = 0;
  cudaEvent_t stage_ev = nullptr;
  ~otm_server() {
    for (auto& ln : lanes) {
      if (ln.stream) cudaStreamSynchronize(ln.stream);
      ln.cache.clear();  // buffers go back to the pool on the lane's stream
      if (ln.stream) {
        cudaStreamSynchronize(ln.stream);
        cudaStreamDestroy(ln.stream);
      }
      if (ln.done) cudaEventDestroy(ln.done);
      if (ln.stage) cudaFreeHost(ln.stage);
    }
    if (stream) cudaStreamSynchronize(stream);
    reqs.clear();
    if (stream) cudaStreamSynchronize(stream);
    if (d_desc) cudaFree(d_desc);
    if (d_tasks) cudaFree(d_tasks);
    if (d_slots) cudaFree(d_slots);
    if (d_status) cudaFree(d_status);
    if (h_status) cudaFreeHost(h_status);
    if (h_stage) cudaFreeHost(h_stage);
    if (stage_ev) cudaEventDestroy(stage_ev);
    if (pool) cudaMemPoolDestroy(pool);
  }
};

namespace otm {

// The request's host copy of its field is no longer needed (uploaded, or never will be).
static void release_field(otm_server* s, Request& r) {
  if (r.pinned) s->ring.release(r.ring_seq);
  r.pinned = nullptr;
  r.ring_seq = -1;
  r.k.clear();
  r.k.shrink_to_fit();
}

// A request leaves the device: its buffers go back to the pool (stream-ordered).
static void release(otm_server* s, Request& r) {
  if (r.slot >= 0) s->slots[r.slot] = -1;
  r.slot = -1;
  r.h.reset();
  s->bytes_in_use -= std::min(s->bytes_in_use, r.bytes);
}

static otm_status admit(otm_server* s, Request& r, int slot) {
  otm_config c;
  homo_config(s->cfg, r.reso, &c);
  r.h.reset(new (std::nothrow) Homo());
  if (!r.h) return OTM_ERR_OUT_OF_MEMORY;
  Homo& H = *r.h;
  OTM_TRY(H.build(c, s->stream, s->pool, true));
  const Dims d0 = H.lv[0].d;
  const size_t nv = d0.nv();
  float* kdev = nullptr;
  OTM_CUDA(cudaMallocFromPoolAsync((void**)&kdev, nv * sizeof(float), s->pool, s->stream));
  if (s->stage_used + nv > s->stage_cap) return OTM_ERR_STATE;  // sized by the caller
  float* stg = s->h_stage + s->stage_used;
  s->stage_used += nv;
  std::memcpy(stg, r.field(), nv * sizeof(float));
  release_field(s, r);
  OTM_CUDA(cudaMemcpyAsync(kdev, stg, nv * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  otm_status st = H.update(kdev, d0.nx);
  cudaFreeAsync(kdev, s->stream);
  OTM_TRY(st);
  OTM_TRY(H.join_coarse());  // the batched kernels read the coarse stencils directly
  H.launch_solve_init();
  // descriptor of the request for the batched kernels
  ReqDesc D;
  std::memset(&D, 0, sizeof(D));
  const int L = int(H.lv.size());
  int tl = -1;
  for (int l = 1; l < L; l++)
    if (H.lv[l].d.nv() <= size_t(kTailMaxNv)) {
      tl = l;
      break;
    }
  if (H.face) {
    set_error("serving needs the cube element (no edge-neighbour coupling)");
    return OTM_ERR_UNSUPPORTED;
  }
  if (tl < 0 || L > kSrvMaxLevels) {
    set_error("serving needs a cell with at least two multigrid levels");
    return OTM_ERR_UNSUPPORTED;
  }
  D.nlev = L;
  D.tail_l = tl;
  D.nc = H.nc;
  for (int l = 0; l < L; l++) D.lv[l] = ReqLevel{H.lv[l].d, H.lv[l].u, H.lv[l].f, H.lv[l].r, H.lv[l].st};
  D.ks = H.ks;
  D.x = H.x;
  D.p = H.p;
  D.q = H.q;
  D.partials = H.partials;
  D.sc = H.sc;
  D.op = H.op;
  TailDesc& td = D.tail;
  td.nlev = L - tl;
  td.pre = c.pre_smooth;
  td.post = c.post_smooth;
  td.nc = H.nc;
  int off = 0;
  for (int i = 0; i < td.nlev; i++) {
    td.lv[i].d = H.lv[tl + i].d;
    td.lv[i].st = H.lv[tl + i].st;
    td.lv[i].off = off;
    off += int(9 * H.lv[tl + i].d.nv());
  }
  td.f_in = H.lv[tl].f;
  td.u_out = H.lv[tl].u;
  td.Ainv = H.Ainv;
  OTM_CUDA(cudaMemcpyAsync(s->d_desc + slot, &D, sizeof(ReqDesc), cudaMemcpyHostToDevice, s->stream));
  r.slot = slot;
  s->slots[slot] = r.id;
  r.state = 1;
  r.info.admit_s = now_s();
  return OTM_OK;
}

struct Segment {
  size_t off = 0;
  int n = 0;
  int blocks = 0;
};

// Append one task per participating slot; blocks(nv of that level) gives the block count.
template <typename F>
static Segment make_segment(std::vector<BTask>& all, const std::vector<std::pair<int, const Homo*>>& part, int level,
                            F blocks) {
  Segment sg;
  sg.off = all.size();
  int b0 = 0;
  for (auto& pr : part) {
    const int nb = blocks(pr.second, level);
    all.push_back(BTask{pr.first, level, b0, nb});
    b0 += nb;
  }
  sg.n = int(part.size());
  sg.blocks = b0;
  return sg;
}

// Run iters batched preconditioned-CG iterations over the running slots.
static otm_status run_batch(otm_server* s, const std::vector<int>& run_slots, int iters) {
  std::vector<std::pair<int, const Homo*>> all;
  int Lmax = 0;
  size_t tail_smem = 0;
  for (int sl : run_slots) {
    const Homo* H = s->reqs[s->slots[sl]].h.get();
    all.emplace_back(sl, H);
    int tl = 1;
    while (H->lv[tl].d.nv() > size_t(kTailMaxNv)) tl++;
    Lmax = std::max(Lmax, tl);
    size_t sm = 0;
    for (size_t l = tl; l < H->lv.size(); l++) sm += 9 * H->lv[l].d.nv() * sizeof(float);
    tail_smem = std::max(tail_smem, sm);
  }
  auto tail_of = [](const Homo* H) {
    int tl = 1;
    while (H->lv[tl].d.nv() > size_t(kTailMaxNv)) tl++;
    return tl;
  };
  std::vector<BTask> tasks;
  std::vector<Segment> zero(Lmax), gs(Lmax), res(Lmax), rst(Lmax), pro(Lmax);
  auto cdiv = [](size_t a) { return int((a + kBlock - 1) / kBlock); };
  for (int l = 0; l < Lmax; l++) {
    std::vector<std::pair<int, const Homo*>> part;
    for (auto& pr : all)
      if (l < tail_of(pr.second)) part.push_back(pr);
    zero[l] = make_segment(tasks, part, l, [&](const Homo* H, int lv) { return cdiv(3 * H->lv[lv].d.nv()); });
    gs[l] = make_segment(tasks, part, l, [&](const Homo* H, int lv) { return cdiv(H->lv[lv].d.nv() >> 3); });
    res[l] = make_segment(tasks, part, l, [&](const Homo* H, int lv) { return cdiv(H->lv[lv].d.nv()); });
    rst[l] = make_segment(tasks, part, l, [&](const Homo* H, int lv) { return cdiv(H->lv[lv + 1].d.nv()); });
    pro[l] = make_segment(tasks, part, l, [&](const Homo* H, int lv) { return cdiv(H->lv[lv].d.nv()); });
  }
  const Segment tail = make_segment(tasks, all, 0, [](const Homo*, int) { return 1; });
  const Segment red = make_segment(tasks, all, 0, [](const Homo* H, int) { return reduce_blocks(H->lv[0].d.nv()); });
  const Segment el0 = make_segment(tasks, all, 0, [&](const Homo* H, int) { return cdiv(H->lv[0].d.nv()); });
  if (tasks.size() > s->task_cap) {
    if (s->d_tasks) cudaFreeAsync(s->d_tasks, s->stream);
    s->task_cap = tasks.size() * 2;
    OTM_CUDA(scratch_malloc((void**)&s->d_tasks, s->task_cap * sizeof(BTask), s->stream));
  }
  OTM_CUDA(cudaMemcpyAsync(s->d_tasks, tasks.data(), tasks.size() * sizeof(BTask), cudaMemcpyHostToDevice, s->stream));
  OTM_CUDA(cudaFuncSetAttribute(kb_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem));
  const ReqDesc* R = s->d_desc;
  const int pre = s->cfg.pre_smooth, post = s->cfg.pre_smooth;
  auto T = [&](const Segment& sg) { return s->d_tasks + sg.off; };
  uint64_t launches = 0;
  for (int it = 0; it < iters; it++) {
    for (int l = 0; l < Lmax; l++) {
      if (!gs[l].n) continue;
      const int passes = l == 0 ? 4 : 8;  // colour pairs on the fine level
      kb_zero<<<zero[l].blocks, kBlock, 0, s->stream>>>(T(zero[l]), zero[l].n, R);
      for (int sw = 0; sw < pre; sw++)
        for (int c = 0; c < passes; c++) kb_gs<<<gs[l].blocks, kBlock, 0, s->stream>>>(T(gs[l]), gs[l].n, R, c);
      kb_resid<<<res[l].blocks, kBlock, 0, s->stream>>>(T(res[l]), res[l].n, R);
      kb_restrict<<<rst[l].blocks, kBlock, 0, s->stream>>>(T(rst[l]), rst[l].n, R);
      launches += 3 + passes * pre;
    }
    kb_tail<<<tail.blocks, kTailThreads, tail_smem, s->stream>>>(T(tail), tail.n, R);
    launches++;
    for (int l = Lmax - 1; l >= 0; l--) {
      if (!gs[l].n) continue;
      const int passes = l == 0 ? 4 : 8;
      kb_prolong<<<pro[l].blocks, kBlock, 0, s->stream>>>(T(pro[l]), pro[l].n, R);
      for (int sw = 0; sw < post; sw++)
        for (int c = passes - 1; c >= 0; c--) kb_gs<<<gs[l].blocks, kBlock, 0, s->stream>>>(T(gs[l]), gs[l].n, R, c);
      launches += 1 + passes * post;
    }
    kb_dot_rz<<<red.blocks, kBlock, 0, s->stream>>>(T(red), red.n, R);
    kb_update_p<<<el0.blocks, kBlock, 0, s->stream>>>(T(el0), el0.n, R);
    kb_apply_dot<<<red.blocks, kBlock, 0, s->stream>>>(T(red), red.n, R);
    kb_update_xr<<<red.blocks, kBlock, 0, s->stream>>>(T(red), red.n, R, s->cfg.max_iter);
    launches += 4;
  }
  OTM_CHECK_LAUNCH("batched iteration");
  count_launches(launches);
  return OTM_OK;
}

static otm_status gather(otm_server* s, const std::vector<int>& sl) {
  if (sl.empty()) return OTM_OK;
  OTM_CUDA(cudaMemcpyAsync(s->d_slots, sl.data(), sl.size() * sizeof(int), cudaMemcpyHostToDevice, s->stream));
  kb_gather<<<ceil_div(sl.size(), 128), 128, 0, s->stream>>>(s->d_slots, int(sl.size()), s->d_desc, s->d_status);
  count_launches(1);
  OTM_CUDA(cudaMemcpyAsync(s->h_status, s->d_status, sl.size() * sizeof(SlotStatus), cudaMemcpyDeviceToHost,
                           s->stream));
  OTM_CUDA(cudaStreamSynchronize(s->stream));
  return OTM_OK;
}

// ---------------------------------------------------------------------------------------
// Handle form
// ---------------------------------------------------------------------------------------
static bool same_reso(const int a[3], const int b[3]) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; }

static void finish_request(otm_server* s, Request& r, otm_status st, bool have_result, const double kh[6]) {
  if (r.cancel) {
    r.state = 3;
    r.status = OTM_ERR_CANCELLED;
  } else {
    if (have_result) {
      int cnt = 0;
      for (int a = 0; a < 3; a++)
        for (int b = a; b < 3; b++) {
          r.C[a * 3 + b] = kh[cnt];
          r.C[b * 3 + a] = kh[cnt];
          cnt++;
        }
    }
    r.status = st;
    r.state = (have_result && (st == OTM_OK || st == OTM_ERR_NOT_CONVERGED)) ? 2 : 4;
  }
  r.info.stats.status = st;
  r.info.done_s = now_s();
  s->bytes_in_use -= std::min(s->bytes_in_use, r.bytes);
  release_field(s, r);
}

// The lane's request has passed its event: status, statistics and K^H from pinned memory.
static void retire_lane(otm_server* s, Lane& ln) {
  Request& r = s->reqs[ln.req];
  Homo& H = *ln.run;
  const SolveScalars& S = *H.sc_host;
  otm_status st = H.check_flags();
  count_launches(1 + H.loop_body_kernels * uint64_t(S.loop));
  r.info.stats.iterations = S.iter;
  for (int c = 0; c < 3; c++) r.info.stats.rel_res[c] = S.relres[c];
  r.info.stats.levels = int(H.lv.size());
  r.info.stats.cluster_level = H.cluster_l;
  for (int i = 0; i < 3; i++) r.info.stats.coarsest_reso[i] = H.stats.coarsest_reso[i];
  if (st == OTM_OK) {
    if (S.nan)
      st = OTM_ERR_DIVERGED;
    else
      for (int c = 0; c < 3; c++)
        if (!(S.relres[c] <= s->cfg.fem_rel_thres)) st = OTM_ERR_NOT_CONVERGED;
  }
  finish_request(s, r, st, st == OTM_OK || st == OTM_ERR_NOT_CONVERGED, S.kh);
  ln.req = -1;
  ln.run = nullptr;
}

static otm_status retire_finished(otm_server* s, bool* any) {
  for (Lane& ln : s->lanes) {
    if (ln.req < 0) continue;
    const cudaError_t e = cudaEventQuery(ln.done);
    if (e == cudaErrorNotReady) continue;
    if (e != cudaSuccess) return cuda_fail(e, "serving lane");
    retire_lane(s, ln);
    *any = true;
  }
  return OTM_OK;
}

static void drop_handle(otm_server* s, Lane& ln, size_t i) {
  s->bytes_resident -= std::min(s->bytes_resident, ln.cache[i].bytes);
  ln.cache.erase(ln.cache.begin() + i);
}

// Make room for `need` more resident bytes by destroying idle handles, least recently used
// first. Returns false (destroying nothing) when even all idle handles would not be enough.
static bool make_room(otm_server* s, size_t need) {
  const size_t budget = s->cfg.hbm_budget_bytes;
  if (s->bytes_resident + need <= budget) return true;
  size_t idle = 0;
  for (Lane& ln : s->lanes)
    for (auto& c : ln.cache)
      if (c.h.get() != ln.run) idle += c.bytes;
  if (s->bytes_resident - std::min(s->bytes_resident, idle) + need > budget) return false;
  while (s->bytes_resident + need > budget) {
    Lane* best_lane = nullptr;
    size_t best = 0;
    uint64_t oldest = UINT64_MAX;
    for (Lane& ln : s->lanes)
      for (size_t i = 0; i < ln.cache.size(); i++)
        if (ln.cache[i].h.get() != ln.run && ln.cache[i].last_use < oldest) {
          oldest = ln.cache[i].last_use;
          best_lane = &ln;
          best = i;
        }
    if (!best_lane) return false;
    drop_handle(s, *best_lane, best);
  }
  return true;
}

static void handle_config(const otm_server_config& sc, const int reso[3], otm_config* c) {
  homo_config(sc, reso, c);
  c->use_graphs = 1;  // the iteration loop as one device-side graph launch
  c->warm_start = 0;  // every request from a zero initial guess
}

// Queue the whole request on the lane: field upload, operator setup, solve, K^H, scalars back.
static otm_status launch_on_lane(otm_server* s, Request& r, Lane& ln, size_t ci) {
  CachedHandle& ch = ln.cache[ci];
  Homo& H = *ch.h;
  const size_t nv = size_t(r.reso[0]) * r.reso[1] * r.reso[2];
  if (!r.pinned && nv > ln.stage_cap) {
    if (ln.stage) cudaFreeHost(ln.stage);
    ln.stage = nullptr;
    ln.stage_cap = 0;
    OTM_CUDA(cudaMallocHost((void**)&ln.stage, nv * sizeof(float)));
    ln.stage_cap = nv;
  }
  const float* src = r.pinned;  // uploaded straight from the ring, released at retirement
  if (!src) {
    std::memcpy(ln.stage, r.k.data(), nv * sizeof(float));  // the lane is idle: its last copy is done
    src = ln.stage;
  }
  // the right-hand-side buffer holds the field until the solve start overwrites it
  OTM_CUDA(cudaMemcpyAsync(H.b, src, nv * sizeof(float), cudaMemcpyHostToDevice, ln.stream));
  OTM_TRY(H.update(H.b, r.reso[0]));
  OTM_CUDA(cudaMemsetAsync(H.x, 0, 3 * nv * sizeof(float), ln.stream));
  OTM_TRY(H.launch_device_solve(true));
  OTM_CUDA(cudaEventRecord(ln.done, ln.stream));
  ln.req = r.id;
  ln.run = &H;
  ch.last_use = ++s->use_clock;
  return OTM_OK;
}

// Admit queued requests, first come first served, onto idle lanes while the budget allows.
static otm_status admit_handles(otm_server* s, bool* any) {
  while (!s->queue.empty()) {
    const int64_t id = s->queue.front();
    Request& r = s->reqs[id];
    if (r.cancel) {
      s->queue.pop_front();
      r.state = 3;
      r.status = OTM_ERR_CANCELLED;
      r.info.done_s = now_s();
      release_field(s, r);
      *any = true;
      continue;
    }
    // an idle lane that already holds a handle of this size, else the idle lane holding the
    // fewest handles
    Lane* lane = nullptr;
    int ci = -1;
    for (Lane& ln : s->lanes) {
      if (ln.req >= 0) continue;
      for (size_t i = 0; i < ln.cache.size(); i++)
        if (same_reso(ln.cache[i].reso, r.reso)) {
          lane = &ln;
          ci = int(i);
          break;
        }
      if (lane) break;
    }
    if (!lane)
      for (Lane& ln : s->lanes)
        if (ln.req < 0 && (!lane || ln.cache.size() < lane->cache.size())) lane = &ln;
    if (!lane) break;  // every lane is busy
    if (ci < 0 && !make_room(s, r.bytes)) break;  // the head of the queue waits for memory
    s->queue.pop_front();
    *any = true;
    s->bytes_in_use += r.bytes;
    r.state = 1;
    r.info.admit_s = now_s();
    if (ci < 0) {
      CachedHandle ch;
      for (int i = 0; i < 3; i++) ch.reso[i] = r.reso[i];
      ch.bytes = r.bytes;
      ch.h.reset(new (std::nothrow) Homo());
      otm_status bst = OTM_ERR_OUT_OF_MEMORY;
      if (ch.h) {
        otm_config c;
        handle_config(s->cfg, r.reso, &c);
        bst = ch.h->build(c, lane->stream, s->pool, true);
      }
      if (bst != OTM_OK) {
        finish_request(s, r, bst, false, nullptr);
        continue;
      }
      lane->cache.push_back(std::move(ch));
      s->bytes_resident += r.bytes;
      ci = int(lane->cache.size()) - 1;
    }
    const otm_status st = launch_on_lane(s, r, *lane, size_t(ci));
    if (st != OTM_OK) {
      // nothing of the request may still run when its handle goes: wait for the lane
      cudaStreamSynchronize(lane->stream);
      lane->req = -1;
      lane->run = nullptr;
      drop_handle(s, *lane, size_t(ci));
      finish_request(s, r, st, false, nullptr);
      if (st == OTM_ERR_CUDA) return st;
    }
  }
  return OTM_OK;
}

static otm_status step_handles(otm_server* s) {
  const double deadline = now_s() + 600.0;
  while (true) {
    bool retired = false, admitted = false;
    OTM_TRY(retire_finished(s, &retired));
    OTM_TRY(admit_handles(s, &admitted));
    bool running = false;
    for (Lane& ln : s->lanes) running |= ln.req >= 0;
    // return at once unless the queue is blocked behind running requests
    if (retired || admitted || s->queue.empty() || !running) return OTM_OK;
    if (now_s() > deadline) {
      set_error("no serving lane finished within 600 s");
      return OTM_ERR_TIMEOUT;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

}  // namespace otm

extern "C" {

otm_status otm_server_config_init(otm_server_config* cfg) {
  if (!cfg) return OTM_ERR_INVALID_ARGUMENT;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->hbm_budget_bytes = size_t(150) * 1000 * 1000 * 1000;
  cfg->max_active = 64;
  cfg->fem_rel_thres = 1e-6;
  cfg->max_iter = 200;
  cfg->pre_smooth = 2;
  cfg->iters_per_step = 2;
  cfg->power_penal = 1.0f;
  cfg->batched = 0;
  cfg->streams = 8;
  cfg->host_stage_bytes = size_t(1) << 30;
  return OTM_OK;
}

size_t otm_server_request_bytes(const int reso[3]) {
  if (!reso) return 0;
  return otm::request_bytes(reso);
}

otm_status otm_server_create(const otm_server_config* cfg, void* stream, otm_server** out) {
  if (!cfg || !out || cfg->max_active < 1 || cfg->max_active > kSrvMaxActive || cfg->pre_smooth < 1 ||
      cfg->iters_per_step < 1 || cfg->max_iter < 1 || !(cfg->fem_rel_thres > 0) ||
      (!cfg->batched && (cfg->streams < 1 || cfg->streams > kSrvMaxStreams)))
    return OTM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::unique_ptr<otm_server> s(new (std::nothrow) otm_server());
  if (!s) return OTM_ERR_OUT_OF_MEMORY;
  s->cfg = *cfg;
  s->stream = (cudaStream_t)stream;
  int dev = 0;
  OTM_CUDA(cudaGetDevice(&dev));
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  OTM_CUDA(cudaMemPoolCreate(&s->pool, &props));
  uint64_t keep = cfg->hbm_budget_bytes;  // keep freed request memory for the next admissions
  OTM_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  s->slots.assign(cfg->max_active, -1);
  OTM_CUDA(cudaMalloc((void**)&s->d_desc, sizeof(ReqDesc) * cfg->max_active));
  OTM_CUDA(cudaMalloc((void**)&s->d_slots, sizeof(int) * cfg->max_active));
  OTM_CUDA(cudaMalloc((void**)&s->d_status, sizeof(SlotStatus) * cfg->max_active));
  OTM_CUDA(cudaMallocHost((void**)&s->h_status, sizeof(SlotStatus) * cfg->max_active));
  OTM_CUDA(s->ring.init(cfg->host_stage_bytes));
  s->handles = !cfg->batched;
  if (s->handles) {
    s->lanes.resize(std::min(cfg->streams, cfg->max_active));
    for (Lane& ln : s->lanes) {
      OTM_CUDA(cudaStreamCreateWithFlags(&ln.stream, cudaStreamNonBlocking));
      OTM_CUDA(cudaEventCreateWithFlags(&ln.done, cudaEventDisableTiming));
    }
  }
  *out = s.release();
  return OTM_OK;
}

otm_status otm_server_destroy(otm_server* s) {
  if (!s) return OTM_ERR_INVALID_ARGUMENT;
  delete s;
  return OTM_OK;
}

otm_status otm_server_submit(otm_server* s, const int reso[3], const float* k_host, int64_t* request_id) {
  if (!s || !reso || !k_host || !request_id) return OTM_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < 3; i++)
    if (reso[i] < 8 || reso[i] > 1024) {
      set_error("serving supports 8 to 1024 cells per axis");
      return OTM_ERR_UNSUPPORTED;
    }
  const size_t bytes = request_bytes(reso);
  if (bytes > s->cfg.hbm_budget_bytes) {
    set_error("request larger than the serving memory budget");
    return OTM_ERR_BUDGET;
  }
  const size_t nv = size_t(reso[0]) * reso[1] * reso[2];
  Request r;
  r.id = s->next_id++;
  for (int i = 0; i < 3; i++) r.reso[i] = reso[i];
  r.pinned = s->ring.alloc(nv, &r.ring_seq);
  if (r.pinned)
    std::memcpy(r.pinned, k_host, nv * sizeof(float));
  else
    r.k.assign(k_host, k_host + nv);
  r.bytes = bytes;
  r.info.submit_s = now_s();
  r.info.state = 0;
  const int64_t id = r.id;
  s->reqs.emplace(id, std::move(r));
  s->queue.push_back(id);
  *request_id = id;
  return OTM_OK;
}

otm_status otm_server_step(otm_server* s, int* n_running, int* n_queued) {
  if (!s) return OTM_ERR_INVALID_ARGUMENT;
  if (s->handles) {
    const otm_status st = step_handles(s);
    int nr = 0;
    for (const Lane& ln : s->lanes) nr += ln.req >= 0;
    if (n_running) *n_running = nr;
    if (n_queued) *n_queued = int(s->queue.size());
    return st;
  }
  // 1. cancelled requests leave
  for (int sl = 0; sl < int(s->slots.size()); sl++) {
    const int64_t id = s->slots[sl];
    if (id < 0) continue;
    Request& r = s->reqs[id];
    if (r.cancel) {
      release(s, r);
      r.state = 3;
      r.status = OTM_ERR_CANCELLED;
      r.info.done_s = now_s();
    }
  }
  // 2. admit queued requests while a slot and the budget allow (first come, first served)
  {
    // the staging area is free once the previous admissions' copies have completed
    if (s->stage_ev) OTM_CUDA(cudaEventSynchronize(s->stage_ev));
    s->stage_used = 0;
    size_t need = 0, used_bytes = s->bytes_in_use;
    int free_slots = 0;
    for (int64_t id : s->slots) free_slots += id < 0;
    for (int64_t id : s->queue) {
      const Request& r = s->reqs[id];
      if (free_slots == 0 || used_bytes + r.bytes > s->cfg.hbm_budget_bytes) break;
      need += size_t(r.reso[0]) * r.reso[1] * r.reso[2];
      used_bytes += r.bytes;
      free_slots--;
    }
    if (need > s->stage_cap) {
      if (s->h_stage) cudaFreeHost(s->h_stage);
      s->h_stage = nullptr;
      s->stage_cap = std::max(need, s->stage_cap * 2);
      OTM_CUDA(cudaMallocHost((void**)&s->h_stage, s->stage_cap * sizeof(float)));
    }
    if (!s->stage_ev) OTM_CUDA(cudaEventCreateWithFlags(&s->stage_ev, cudaEventDisableTiming));
  }
  while (!s->queue.empty()) {
    const int64_t id = s->queue.front();
    Request& r = s->reqs[id];
    if (r.cancel) {
      s->queue.pop_front();
      r.state = 3;
      r.status = OTM_ERR_CANCELLED;
      r.info.done_s = now_s();
      release_field(s, r);
      continue;
    }
    int slot = -1;
    for (int i = 0; i < int(s->slots.size()); i++)
      if (s->slots[i] < 0) {
        slot = i;
        break;
      }
    if (slot < 0 || s->bytes_in_use + r.bytes > s->cfg.hbm_budget_bytes) break;
    s->queue.pop_front();
    s->bytes_in_use += r.bytes;
    otm_status st = admit(s, r, slot);
    if (st != OTM_OK) {
      release(s, r);
      r.state = 4;
      r.status = st;
      r.info.done_s = now_s();
      release_field(s, r);
    }
  }
  if (s->stage_used) OTM_CUDA(cudaEventRecord(s->stage_ev, s->stream));
  // 3. advance every running request
  std::vector<int> run;
  for (int sl = 0; sl < int(s->slots.size()); sl++)
    if (s->slots[sl] >= 0) run.push_back(sl);
  if (!run.empty()) {
    OTM_TRY(run_batch(s, run, s->cfg.iters_per_step));
    OTM_TRY(gather(s, run));
    // 4. finished requests: K^H, results, memory back to the pool
    std::vector<int> fin;
    for (size_t i = 0; i < run.size(); i++)
      if (s->h_status[i].done) fin.push_back(run[i]);
    if (!fin.empty()) {
      for (int sl : fin) s->reqs[s->slots[sl]].h->launch_heat_matrix();
      OTM_TRY(gather(s, fin));
      for (size_t i = 0; i < fin.size(); i++) {
        Request& r = s->reqs[s->slots[fin[i]]];
        const SlotStatus& ss = s->h_status[i];
        int cnt = 0;
        for (int a = 0; a < 3; a++)
          for (int b = a; b < 3; b++) {
            r.C[a * 3 + b] = ss.kh[cnt];
            r.C[b * 3 + a] = ss.kh[cnt];
            cnt++;
          }
        r.info.stats.iterations = ss.iter;
        for (int c = 0; c < 3; c++) r.info.stats.rel_res[c] = ss.relres[c];
        r.info.stats.levels = int(r.h->lv.size());
        otm_status st = OTM_OK;
        if (ss.nan)
          st = OTM_ERR_DIVERGED;
        else
          for (int c = 0; c < 3; c++)
            if (!(ss.relres[c] <= s->cfg.fem_rel_thres)) st = OTM_ERR_NOT_CONVERGED;
        r.info.stats.status = st;
        r.status = st;
        r.state = (st == OTM_OK || st == OTM_ERR_NOT_CONVERGED) ? 2 : 4;
        r.info.done_s = now_s();
        release(s, r);
        release_field(s, r);
      }
    }
  }
  int nr = 0;
  for (int64_t id : s->slots) nr += id >= 0;
  if (n_running) *n_running = nr;
  if (n_queued) *n_queued = int(s->queue.size());
  return OTM_OK;
}

otm_status otm_server_poll(otm_server* s, int64_t request_id, double C[9], otm_request_info* info) {
  if (!s) return OTM_ERR_INVALID_ARGUMENT;
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return OTM_ERR_INVALID_ARGUMENT;
  Request& r = it->second;
  if (info) {
    *info = r.info;
    info->state = r.state;
    info->status = r.status;
  }
  if (r.state <= 1) return OTM_ERR_NOT_READY;
  if (C && r.state == 2) std::memcpy(C, r.C, sizeof(r.C));
  return otm_status(r.status);
}

otm_status otm_server_cancel(otm_server* s, int64_t request_id) {
  if (!s) return OTM_ERR_INVALID_ARGUMENT;
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return OTM_ERR_INVALID_ARGUMENT;
  if (it->second.state <= 1) it->second.cancel = true;
  return OTM_OK;
}

size_t otm_server_bytes_in_use(const otm_server* s) { return s ? s->bytes_in_use : 0; }

size_t otm_server_bytes_resident(const otm_server* s) {
  if (!s) return 0;
  return s->handles ? s->bytes_resident : s->bytes_in_use;
}

}  // extern "C"
