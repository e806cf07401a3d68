// Persistent mixed-scheme, mixed-operation batch: one launch of 2 CTAs per SM that pull
// tasks from a device work queue until it is empty.
//
// A request is one KEM operation (FrodoKEM-976 or Saber l = 2/3/4; keypair, encaps or
// decaps) on caller device buffers.  Each operation is a short chain of stages (the same
// per-instance / per-CTA routines the batched kernels use): thread-level stages (hash
// chains, XOF prologues) run up to 256 instances per task, one per thread; CTA-level
// stages (Frodo A-generation + product, Saber products, Frodo W) run one instance per
// task.  The host orders the task list by simulating list scheduling on the GPU's CTA
// slots (so every task is preceded by the tasks it depends on) and each task waits, with
// a bounded spin, for its instances' previous stages through per-request stage counters
// (release: __threadfence + atomicAdd; acquire: ld.acquire.gpu).
//
// This translation unit is compiled with -Xptxas -dlcm=cg: global loads bypass L1, because
// L1 is not coherent within a launch and requests may share 128-byte lines that a later
// stage of a neighbouring request is still writing.
//
// The reference has no equivalent: each of its operations is a fixed chain of launches
// over a compile-time batch of one scheme (FrodoKEM976-GPU/src/cuda_kernel.cu,
// SABER-GPU/src/cuda_kernel.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <queue>
#include <vector>

#include "mixed_dev.cuh"

namespace dpkem {
namespace mixed {
namespace {

struct Task {
  uint16_t code;
  uint16_t count;
  uint32_t first;  // index into idx[]
};

struct Plan {
  const DevReq *req;
  const Task *tasks;
  const uint32_t *idx;
  uint32_t ntasks;
  uint32_t *head;
  uint32_t *done;
  uint32_t *err;
  CoinKey key;  // coin stream key of requests with gen set
};

// Wait limit for a dependency: a dependency was fetched earlier and is running, so a
// healthy wait is at most one task (milliseconds).  After any error every wait returns at
// once, so a broken plan drains instead of accumulating timeouts.
constexpr uint64_t kDepLimitNs = 2000000000ull;

// true when request r has completed `need` stage roles; false on expiry (the error word is
// set) or when an error is already recorded, in which case the caller skips its stage.
__device__ __forceinline__ bool wait_done(const Plan &p, uint32_t r, uint32_t need) {
  if (ld_relaxed(p.done + r) < need) {
    const uint64_t t0 = globaltimer_ns();
    while (ld_relaxed(p.done + r) < need) {
      if (ld_relaxed(p.err) != 0) return false;
      __nanosleep(200);
      if (globaltimer_ns() - t0 > kDepLimitNs) {
        atomicOr(p.err, DEV_ERR_TIMEOUT);
        return false;
      }
    }
  }
  __threadfence();  // acquire side of mark_done's release
  return true;
}

__device__ __forceinline__ void mark_done(const Plan &p, uint32_t r) {
  __threadfence();
  atomicAdd(p.done + r, 1u);
}

__global__ void __launch_bounds__(256, 2) mixed_kernel(Plan p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint32_t s_task, s_tmem, s_ready;
  const int tid = threadIdx.x;
  if (tid < 32) {
    tmem_alloc(&s_tmem, fdev::TC_TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = s_tmem;
  while (true) {
    if (tid == 0) s_task = atomicAdd(p.head, 1u);
    __syncthreads();
    const uint32_t t = s_task;
    __syncthreads();
    if (t >= p.ntasks) break;
    const Task tk = p.tasks[t];
    const int code = tk.code & (kWarpTask - 1), scheme = scheme_of(code), op = op_of(code), stage = stage_of(code);
    const int kind = kind_of(scheme, op, stage);
    const uint32_t need = threshold(scheme, op, stage);
    if (kind == K_CTA) {
      const uint32_t r = p.idx[tk.first];
      if (tid == 0) s_ready = wait_done(p, r, need) ? 1u : 0u;
      __syncthreads();
      if (s_ready) cta_stage(code, p.req[r], smem, tbase, p.err);  // skipped after an error: the batch drains
      __syncthreads();
      if (tid == 0) mark_done(p, r);
    } else if (tk.code & kWarpTask) {
      const int warp = tid >> 5, lane = tid & 31;
      const int slot = kind == K_THREAD2 ? warp >> 1 : warp, role = kind == K_THREAD2 ? warp & 1 : 0;
      if (slot < tk.count) {  // warp-uniform: every lane of the warp runs the stage
        const uint32_t r = p.idx[tk.first + slot];
        int ok = 0;
        if (lane == 0) ok = wait_done(p, r, need) ? 1 : 0;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok) warp_stage(p.key, code, p.req[r], role);
        __threadfence();  // every lane's writes, before the count that publishes them
        __syncwarp();
        if (lane == 0) atomicAdd(p.done + r, 1u);
      }
    } else {
      const int per = kind == K_THREAD2 ? 128 : 256;
      const int slot = tid % per, role = tid / per;
      if (slot < tk.count) {
        const uint32_t r = p.idx[tk.first + slot];
        if (wait_done(p, r, need)) thread_stage(p.key, code, p.req[r], role);
        mark_done(p, r);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid < 32) {
    tc_fence_after();
    tmem_dealloc(tbase, fdev::TC_TMEM_COLS);
  }
}

// ---------------------------------------------------------------- host: task list
// Estimated CTA-slot time of each stage (microseconds), used only to order tasks.
double est_us(int scheme, int op, int stage, int count) {
  const int kind = kind_of(scheme, op, stage);
  if (scheme <= 1) {
    if (kind == K_CTA) return op == OP_DEC && stage == 0 ? 30.0 : 1700.0;
    const bool prologue = (op == OP_DEC) ? stage == 1 : stage == 0;
    if (!prologue) return 900.0;
    return op == OP_ENC ? 3200.0 : op == OP_DEC ? 2400.0 : 2200.0;
  }
  if (kind == K_CTA) return 60.0;
  if (kind == K_THREAD2) return 250.0;
  (void)count;
  return 120.0;
}

// Tasks of one stage are created in instance order, so a task's dependencies (the previous
// stage's tasks covering its instances) and its dependents are contiguous id ranges.
struct HostTask {
  Task t;
  double dur, ready;
  int pending;       // dependencies not yet scheduled
  int dn_lo, dn_hi;  // dependents [dn_lo, dn_hi]; empty when dn_lo > dn_hi
  int prio;
};

}  // namespace

// Instances per thread-level task (tuning knobs, clamped to what one CTA can hold).
int task_size(int scheme, int kind) {
  const Tuning &t = tuning();
  int v = kind == K_THREAD2 ? t.mixed_pair_task : scheme <= 1 ? t.mixed_frodo_task : t.mixed_thread_task;
  const int cap = kind == K_THREAD2 ? 128 : 256;
  return std::max(1, std::min(v, cap));
}

// Whether a thread-level stage of a group of `count` requests runs as warp tasks (a warp
// per instance), and the instances per task either way.
bool warp_tasks(int kind, size_t count) { return kind != K_CTA && count <= (size_t)tuning().mixed_warp_max; }
int task_per(int scheme, int kind, size_t count) {
  if (kind == K_CTA) return 1;
  if (warp_tasks(kind, count)) return kind == K_THREAD2 ? 4 : 8;
  return task_size(scheme, kind);
}

// Bytes of device memory a plan for these requests needs (tables + scratch records).
size_t plan_bytes(const Req *reqs, size_t n, size_t *ntasks_out) {
  size_t scr = 0, ntasks = 0, nidx = 0;
  size_t counts[5][3] = {};
  for (size_t i = 0; i < n; i++) {
    scr += reqs[i].scheme <= 1 ? kFrodoRec : saber_rec_bytes(reqs[i].scheme);
    counts[reqs[i].scheme][reqs[i].op]++;
  }
  for (int s = 0; s < 5; s++)
    for (int op = 0; op < 3; op++) {
      const size_t c = counts[s][op];
      if (!c) continue;
      for (int st = 0; st < nstages(s, op); st++) {
        const int kind = kind_of(s, op, st);
        const size_t per = (size_t)task_per(s, kind, c);
        ntasks += (c + per - 1) / per;
        nidx += c;
      }
    }
  if (ntasks_out) *ntasks_out = ntasks;
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  return up(n * sizeof(DevReq)) + up(ntasks * sizeof(Task)) + up(nidx * 4) + up(n * 4) + 256 + scr;
}

// Builds the plan in host memory, uploads it into `arena` and returns the launch descriptor.
size_t plan_table_bytes(const Req *reqs, size_t n) {
  size_t ntasks = 0;
  plan_bytes(reqs, n, &ntasks);
  size_t nidx = 0;
  for (size_t i = 0; i < n; i++) nidx += nstages(reqs[i].scheme, reqs[i].op);
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  return up(n * sizeof(DevReq)) + up(ntasks * sizeof(Task)) + nidx * 4;
}

cudaError_t plan_build(const Req *reqs, size_t n, int form, int slots, uint8_t *arena, size_t arena_bytes,
                       uint32_t *err, cudaStream_t st, void *plan_out, const uint8_t *coin_key, uint64_t coin_first,
                       uint8_t *stage, size_t stage_bytes) {
  size_t ntasks = 0;
  const size_t need = plan_bytes(reqs, n, &ntasks);
  if (need > arena_bytes) return cudaErrorMemoryAllocation;
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  std::vector<std::vector<uint32_t>> groups(5 * 3);
  for (size_t i = 0; i < n; i++) groups[reqs[i].scheme * 3 + reqs[i].op].push_back((uint32_t)i);
  size_t nidx = 0;
  for (int g = 0; g < 15; g++)
    if (!groups[g].empty()) nidx += groups[g].size() * nstages(g / 3, g % 3);
  // Host image of the device tables [requests | tasks | idx], uploaded in one copy.
  const size_t o_tasks = up(n * sizeof(DevReq)), o_idx = o_tasks + up(ntasks * sizeof(Task));
  const size_t table = o_idx + nidx * 4;
  std::vector<uint8_t> own;
  uint8_t *img = stage;
  const bool pinned = stage && stage_bytes >= table;
  if (!pinned) {
    own.resize(table);
    img = own.data();
  }
  DevReq *hreq = reinterpret_cast<DevReq *>(img);
  Task *order = reinterpret_cast<Task *>(img + o_tasks);
  uint32_t *idx = reinterpret_cast<uint32_t *>(img + o_idx);
  uint8_t *d_req = arena, *d_tasks = arena + o_tasks, *d_idx = arena + o_idx;
  uint8_t *d_done = d_idx + up(nidx * 4);
  uint8_t *d_head = d_done + up(n * 4);
  uint8_t *d_scr = d_head + 256;

  size_t off = 0;
  for (size_t i = 0; i < n; i++) {
    const Req &r = reqs[i];
    uint8_t *rec = d_scr + off;
    hreq[i] = DevReq{r.scheme, r.op, r.in0, r.in1, r.out0, r.out1, rec, coin_first + i, 0u, 0u};
    if (coin_key && !r.in0 && r.op != OP_DEC) {  // coins drawn on the device into the record
      hreq[i].in0 = rec + (r.scheme <= 1 ? kFrodoCoins : saber_coins_off(r.scheme));
      hreq[i].gen = 1;
    }
    off += r.scheme <= 1 ? kFrodoRec : saber_rec_bytes(r.scheme);
  }
  // Tasks per group and stage; dependencies on the previous stage's tasks are id ranges.
  std::vector<HostTask> ht;
  ht.reserve(ntasks);
  size_t nid = 0;
  std::vector<int> owner_prev, owner;
  for (int g = 0; g < 15; g++) {
    const std::vector<uint32_t> &R = groups[g];
    if (R.empty()) continue;
    const int scheme = g / 3, op = g % 3;
    owner_prev.assign(R.size(), -1);
    owner.assign(R.size(), -1);
    for (int stg = 0; stg < nstages(scheme, op); stg++) {
      const int kind = kind_of(scheme, op, stg);
      const int per = task_per(scheme, kind, R.size());
      const bool warp = warp_tasks(kind, R.size());
      const uint32_t base = (uint32_t)nid;
      std::memcpy(idx + nid, R.data(), R.size() * 4);
      nid += R.size();
      for (size_t a = 0; a < R.size(); a += per) {
        const int cnt = (int)std::min<size_t>(per, R.size() - a);
        const int id = (int)ht.size();
        const int lo = owner_prev[a], hi = owner_prev[a + cnt - 1];
        // a warp per instance runs a sponge chain in about half the time of one thread
        const double dur = est_us(scheme, op, stg, cnt) * (warp ? 0.45 : 1.0);
        const int prio = kind == K_CTA ? (dur > 500 ? 2 : 1) : 0;  // latency-bound thread stages first
        const int code = code_of(scheme, op, stg, form) | (warp ? kWarpTask : 0);
        ht.push_back(HostTask{Task{(uint16_t)code, (uint16_t)cnt, base + (uint32_t)a}, dur,
                              0.0, lo >= 0 ? hi - lo + 1 : 0, INT32_MAX, -1, prio});
        for (int k = 0; k < cnt; k++) owner[a + k] = id;
        for (int d = lo; lo >= 0 && d <= hi; d++) {
          ht[d].dn_lo = std::min(ht[d].dn_lo, id);
          ht[d].dn_hi = std::max(ht[d].dn_hi, id);
        }
      }
      std::swap(owner_prev, owner);
    }
  }
  // List scheduling on `slots` CTA slots: the fetch order is the simulated start order.
  // `waiting` holds tasks whose dependencies are scheduled, keyed by ready time; `ready`
  // holds those whose ready time has passed, keyed by priority then creation order.
  struct ByReady {
    double ready;
    int id;
    bool operator>(const ByReady &o) const { return ready != o.ready ? ready > o.ready : id > o.id; }
  };
  struct ByPrio {
    int prio, id;
    bool operator>(const ByPrio &o) const { return prio != o.prio ? prio > o.prio : id > o.id; }
  };
  std::vector<ByReady> wv;
  std::vector<ByPrio> rv;
  std::vector<double> fv;
  wv.reserve(ht.size());
  rv.reserve(ht.size());
  fv.reserve(std::max(1, slots));
  std::priority_queue<ByReady, std::vector<ByReady>, std::greater<ByReady>> waiting(std::greater<ByReady>(),
                                                                                   std::move(wv));
  std::priority_queue<ByPrio, std::vector<ByPrio>, std::greater<ByPrio>> ready(std::greater<ByPrio>(), std::move(rv));
  std::priority_queue<double, std::vector<double>, std::greater<double>> free_at(std::greater<double>(),
                                                                                 std::move(fv));
  for (int s = 0; s < std::max(1, slots); s++) free_at.push(0.0);
  for (size_t i = 0; i < ht.size(); i++)
    if (ht[i].pending == 0) waiting.push({0.0, (int)i});
  size_t placed = 0;
  while (!waiting.empty() || !ready.empty()) {
    const double w = free_at.top();
    free_at.pop();
    while (!waiting.empty() && waiting.top().ready <= w) {
      ready.push({ht[waiting.top().id].prio, waiting.top().id});
      waiting.pop();
    }
    int id;
    if (!ready.empty()) {
      id = ready.top().id;
      ready.pop();
    } else {
      id = waiting.top().id;
      waiting.pop();
    }
    const double start = std::max(w, ht[id].ready), fin = start + ht[id].dur;
    free_at.push(fin);
    order[placed++] = ht[id].t;
    for (int d = ht[id].dn_lo; d <= ht[id].dn_hi; d++) {
      ht[d].ready = std::max(ht[d].ready, fin);
      if (--ht[d].pending == 0) waiting.push({ht[d].ready, d});
    }
  }
  if (placed != ntasks) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemcpyAsync(d_req, img, table, cudaMemcpyHostToDevice, st);
  // A pageable image must be consumed before the vector goes away; a pinned stage is the
  // caller's to keep until the copy has run.
  if (e == cudaSuccess && !pinned) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  (void)d_tasks;
  Plan *p = static_cast<Plan *>(plan_out);
  *p = Plan{reinterpret_cast<const DevReq *>(d_req), reinterpret_cast<const Task *>(d_tasks),
            reinterpret_cast<const uint32_t *>(d_idx), (uint32_t)ntasks, reinterpret_cast<uint32_t *>(d_head),
            reinterpret_cast<uint32_t *>(d_done), err, default_coin_key()};
  if (coin_key)
    for (int q = 0; q < 4; q++) {
      uint32_t lo, hi;
      std::memcpy(&lo, coin_key + 8 * q, 4);
      std::memcpy(&hi, coin_key + 8 * q + 4, 4);
      p->key.w[q] = make_uint2(lo, hi);
    }
  return cudaSuccess;
}

size_t plan_struct_bytes() { return sizeof(Plan); }

// Grid of the persistent kernel (2 CTAs per SM when they fit); sets its shared-memory limit.
// Call outside stream capture.
cudaError_t kernel_setup(int *grid) {
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem)) != cudaSuccess)
    return e;
  int dev = 0, sms = 0, occ = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mixed_kernel, 256, kSmem);
  *grid = std::max(1, sms * std::max(1, std::min(occ, 2)));
  return cudaSuccess;
}

// Reset the queue and stage counters, then launch the persistent kernel (capturable).
cudaError_t plan_launch(const void *plan, size_t n, int grid, cudaStream_t st) {
  const Plan &p = *static_cast<const Plan *>(plan);
  cudaError_t e;
  if ((e = cudaMemsetAsync(p.done, 0, n * 4, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(p.head, 0, 4, st)) != cudaSuccess) return e;
  mixed_kernel<<<grid, 256, kSmem, st>>>(p);
  return cudaGetLastError();
}

// Response headers of a frame batch (the wire format of dpkem_wire.h): every request's
// header sits 32 bytes before its first input, its response header 32 bytes before its
// first output.  One thread per request copies version, scheme, op and id, writes the
// magic, status OK and the response frame size from resp_bytes[scheme * 3 + op], and
// zeroes the frame's tail padding from payload_end[scheme * 3 + op] on.
struct FrameSizes {
  uint32_t resp_bytes[15];
  uint32_t payload_end[15];
};

__global__ void __launch_bounds__(256) frame_headers_kernel(const DevReq *req, uint32_t n, FrameSizes fs) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevReq r = req[i];
  const uint2 *rq = reinterpret_cast<const uint2 *>(r.in0 - 32);
  const uint2 w0 = rq[0], w1 = rq[1];
  uint4 *rs = reinterpret_cast<uint4 *>(r.out0 - 32);
  // bytes 0-3 magic, 4 version, 5 scheme, 6 op, 7 status (0), 8-15 id, 16-19 frame_bytes
  const int k = r.scheme * 3 + r.op;
  rs[0] = make_uint4(0x464B5044u, w0.y & 0x00FFFFFFu, w1.x, w1.y);
  rs[1] = make_uint4(fs.resp_bytes[k], 0u, 0u, 0u);
  uint8_t *frame = r.out0 - 32;
  for (uint32_t b = fs.payload_end[k]; b < fs.resp_bytes[k]; b++) frame[b] = 0;
}

cudaError_t frame_headers_launch(const void *plan, size_t n, const uint32_t *resp_bytes, const uint32_t *payload_end,
                                 cudaStream_t st) {
  const Plan &p = *static_cast<const Plan *>(plan);
  FrameSizes fs{};
  for (int k = 0; k < 15; k++) {
    fs.resp_bytes[k] = resp_bytes[k];
    fs.payload_end[k] = payload_end[k];
  }
  frame_headers_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p.req, (uint32_t)n, fs);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- diagnostics
// Kernels whose bounded wait cannot be satisfied, to exercise the expiry path end to end.
__global__ void mbar_timeout_kernel(uint32_t *err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // one arrival expected, none ever made
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0)) atomicOr(err, DEV_ERR_TIMEOUT);
}

cudaError_t selftest_timeout(int which, uint8_t *arena, size_t arena_bytes, uint32_t *err, cudaStream_t st) {
  if (which == 0) {
    mbar_timeout_kernel<<<1, 32, 0, st>>>(err);
    return cudaGetLastError();
  }
  // One Saber l=3 encapsulation product task whose prologue never ran: its dependency
  // counter stays 0, the wait expires, the stage is skipped and the kernel exits.
  constexpr size_t kReq = 0, kTask = 256, kIdx = 512, kDone = 768, kHead = 1024, kRec = 2048;
  const size_t kBuf = kRec + ((saber_rec_bytes(3) + 255) & ~(size_t)255);
  if (arena_bytes < kBuf + 4096) return cudaErrorInvalidValue;
  DevReq rq{3, OP_ENC, arena + kBuf, arena + kBuf + 1024, arena + kBuf + 2048, arena + kBuf + 3328,
            arena + kRec, 0, 0u, 0u};
  const Task tk{(uint16_t)code_of(3, OP_ENC, 1, FORM_DP4A), 1, 0};
  std::vector<uint8_t> host(kRec, 0);
  std::memcpy(host.data() + kReq, &rq, sizeof rq);
  std::memcpy(host.data() + kTask, &tk, sizeof tk);
  cudaError_t e = cudaMemcpyAsync(arena, host.data(), host.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // pageable source
  int grid = 0;
  if (e == cudaSuccess) e = kernel_setup(&grid);
  if (e != cudaSuccess) return e;
  const Plan p{reinterpret_cast<const DevReq *>(arena + kReq), reinterpret_cast<const Task *>(arena + kTask),
               reinterpret_cast<const uint32_t *>(arena + kIdx), 1u, reinterpret_cast<uint32_t *>(arena + kHead),
               reinterpret_cast<uint32_t *>(arena + kDone), err, default_coin_key()};
  mixed_kernel<<<1, 256, kSmem, st>>>(p);
  return cudaGetLastError();
}

int slots_for_device() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return 2 * sms;
}

}  // namespace mixed
}  // namespace dpkem
