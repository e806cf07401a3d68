// KEM service: one long-lived persistent launch that takes requests while it runs.
//
// The host appends requests to a ring of request records in device memory and publishes
// the new count (a 4-byte copy, ordered after the records' copy on the same stream).  The
// kernel's CTAs admit them inside the launch: a CTA that sees unadmitted requests claims
// the range and pushes every request into the ready queue of its first stage.  From there
// on a request moves through per-(scheme, operation, stage) ready queues in device memory:
// a CTA with nothing to do claims work from the highest-priority non-empty queue (up to 256
// instances of a thread-level stage, one instance of a CTA-level stage), runs it with the
// stage bodies of the mixed-batch kernel, and pushes each instance on to its next stage's
// queue; the last stage writes the request's ticket into host-mapped memory, which the
// host polls.  Thread-level stages therefore gather ready instances across submissions,
// whatever their arrival time, and no request waits for a launch to drain.
//
// Queues are bounded multi-producer multi-consumer rings of 64-bit entries (sequence << 32
// | request slot), one lap per entry: a producer reserves index j with an atomicAdd on the
// queue's tail and waits for the entry to carry sequence j (its previous lap consumed); a
// consumer claims a range [h, h + k) with a compare-and-swap on the head and waits for
// each entry to carry j + 1 (written).  Entries per queue = request slots, so an entry's
// previous lap is always claimed by a running CTA.  Every wait is bounded: the waits on an
// entry (microseconds when healthy) set the error word after one second; an idle CTA
// sleeps in short steps and the launch ends after `idle_ms` without work (the host
// relaunches it on the next submission) or when the host raises `stop`.
//
// Compiled with -Xptxas -dlcm=cg, like mixed.cu: request records and queue entries change
// during the launch, so global loads must not be served from the non-coherent L1.
//
// The reference has no serving path (FrodoKEM976-GPU/main.cu:13-34, SABER-GPU/main.cu:12-38:
// one fixed batch per program).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/dpkem.h"
#include "ctx.h"
#include "mixed_dev.cuh"

namespace dpkem {
namespace serve {
namespace {

using namespace mixed;

constexpr int kQueues = 60;  // (scheme * 3 + op) * 4 + stage
__host__ __device__ constexpr int queue_of(int scheme, int op, int stage) { return (scheme * 3 + op) * 4 + stage; }
__host__ __device__ constexpr int q_scheme(int q) { return q / 12; }
__host__ __device__ constexpr int q_op(int q) { return (q >> 2) % 3; }
__host__ __device__ constexpr int q_stage(int q) { return q & 3; }
constexpr int kAdmit = 64, kNone = 65, kRetry = 66;

struct alignas(128) Word {
  uint32_t v;
  uint32_t pad[31];
};

// Control words in device memory, each on its own 128-byte line.
struct Ctl {
  Word sub_tail;  // requests published by the host (ticket count mod 2^32)
  Word admitted;  // requests pushed into their first stage's queue
  Word version;   // bumped after every push: idle CTAs watch this word
  Word stop;      // host: end the launch once idle
  Word quit;      // set by the first CTA whose idle limit ran out
  Word err;       // DEV_ERR_* (also mirrored to host_err)
  Word head[kQueues], tail[kQueues];
};

// Counters (device memory, zeroed at open): per queue claims, instances, claims run a warp
// per instance, and thread 0's busy time from claim to hand-off (ns); then the CTAs' idle
// time (ns), admissions, requests admitted and claims lost to another CTA.
constexpr int kStats = kQueues * 4 + 4;

struct Svc {
  Ctl *ctl;
  unsigned long long *stats;  // [kStats]
  const DevReq *req;          // [slots], slot = ticket & qmask
  uint32_t *done;             // [slots] roles finished in the current two-role stage
  unsigned long long *ent;    // [kQueues][slots]
  uint32_t qmask;             // slots - 1 (a power of two)
  uint32_t short_ctas;        // CTAs [0, short_ctas) take only the short-chain queues
  uint32_t warp_max;          // a thread-level backlog up to this runs a warp per instance
  uint32_t nprio, nshort;
  int form;
  uint8_t prio[kQueues];        // queue ids, highest priority first
  uint8_t prio_short[kQueues];  // the same restricted to short-chain (Saber) queues
  uint64_t idle_ns;
  volatile uint32_t *host_done;  // host-mapped [slots]: ticket + 1 once the request completed
  volatile uint32_t *host_err;   // host-mapped error word
  CoinKey key;
};

constexpr uint64_t kEntryWaitNs = 1000000000ull;

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_rel64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void fail(const Svc &p) {
  atomicOr(&p.ctl->err.v, DEV_ERR_TIMEOUT);
  *p.host_err = DEV_ERR_TIMEOUT;
  __threadfence_system();
}

// Waits (bounded) until entry e carries sequence `seq`; its value in *v.
__device__ __forceinline__ bool wait_seq(const Svc &p, const unsigned long long *e, uint32_t seq,
                                         unsigned long long *v) {
  unsigned long long x = ld_relaxed64(e);
  if ((uint32_t)(x >> 32) != seq) {
    const uint64_t t0 = globaltimer_ns();
    do {
      __nanosleep(64);
      x = ld_relaxed64(e);
      if ((uint32_t)(x >> 32) != seq && globaltimer_ns() - t0 > kEntryWaitNs) {
        fail(p);
        return false;
      }
    } while ((uint32_t)(x >> 32) != seq);
  }
  __threadfence();  // acquire side of the entry's release store
  *v = x;
  return true;
}

__device__ __forceinline__ unsigned long long *entry(const Svc &p, int q, uint32_t j) {
  return p.ent + (size_t)q * (p.qmask + 1) + (j & p.qmask);
}

// Appends request slot r to queue q (after this thread's stage writes).  Idle CTAs learn of
// it from the push counter, which the caller bumps once per batch of pushes (wake()).
__device__ __forceinline__ void push(const Svc &p, int q, uint32_t r) {
  __threadfence();
  const uint32_t j = atomicAdd(&p.ctl->tail[q].v, 1u);
  unsigned long long *e = entry(p, q, j);
  unsigned long long x;
  if (wait_seq(p, e, j, &x)) st_rel64(e, ((unsigned long long)(j + 1) << 32) | r);
}

__device__ __forceinline__ void wake(const Svc &p) { atomicAdd(&p.ctl->version.v, 1u); }

// The request slot in claimed entry j of queue q (~0u if the entry never filled); the entry
// is handed to its next lap.
__device__ __forceinline__ uint32_t take(const Svc &p, int q, uint32_t j) {
  unsigned long long *e = entry(p, q, j);
  unsigned long long x;
  if (!wait_seq(p, e, j + 1, &x)) return ~0u;
  st_rel64(e, (unsigned long long)(j + p.qmask + 1) << 32);
  return (uint32_t)x;
}

// Request r finished `stage`: into the next stage's queue, or reported complete.
__device__ __forceinline__ void advance(const Svc &p, int scheme, int op, int stage, uint32_t r) {
  if (stage + 1 < nstages(scheme, op)) {
    push(p, queue_of(scheme, op, stage + 1), r);
    return;
  }
  __threadfence_system();
  p.host_done[r] = p.req[r].ticket + 1u;
}

// One role of a two-role stage finished; the second to finish moves the request on.
__device__ __forceinline__ void role_done(const Svc &p, int scheme, int op, int stage, uint32_t r) {
  __threadfence();
  if (atomicAdd(p.done + r, 1u) == 1u) {
    __threadfence();
    atomicExch(p.done + r, 0u);
    advance(p, scheme, op, stage, r);
  }
}

// CTA-level stages of a few microseconds (the Saber products, FrodoKEM decaps' W): a claim
// may take several instances, run one after another, so that claiming does not cost as
// much as the work.
__host__ __device__ constexpr bool short_cta(int q) {
  return q_scheme(q) >= 2 || (q_op(q) == OP_DEC && q_stage(q) == 0);
}
constexpr uint32_t kCtaBatch = 8;

// Instances one claim takes from queue q with `backlog` ready, and whether they run a warp
// per instance (small backlogs: the chain finishes sooner and the CTA is free again sooner).
__device__ __forceinline__ uint32_t cap_of(const Svc &p, int q, uint32_t backlog, bool *warp) {
  const int kind = kind_of(q_scheme(q), q_op(q), q_stage(q));
  *warp = false;
  if (kind == K_CTA) return short_cta(q) ? min(kCtaBatch, 1u + backlog / 32u) : 1u;
  *warp = backlog <= p.warp_max;
  if (kind == K_THREAD2) return *warp ? 4 : 128;
  return *warp ? 8 : 256;
}

// Warp 0: admission if requests are waiting, else a claim on the highest-priority
// non-empty queue.  Returns the queue (with [*h, *h + *k) claimed), kAdmit (tickets
// [*h, *h + *k) to admit), kNone or kRetry (lost a race).
// *ver, *sub: the push counter and the published count read before looking, so that an
// idle wait on them cannot miss a push made during the scan.
__device__ int pick(const Svc &p, bool short_only, uint32_t *h, uint32_t *k, bool *warp, uint32_t *ver,
                    uint32_t *subp) {
  const int lane = threadIdx.x & 31;
  Ctl *c = p.ctl;
  uint32_t sub = 0, adm = 0, v = 0, quit = 0;
  if (lane == 0) {
    v = ld_relaxed(&c->version.v);
    sub = ld_relaxed(&c->sub_tail.v);
    adm = ld_relaxed(&c->admitted.v);
    quit = ld_relaxed(&c->quit.v);
  }
  *ver = __shfl_sync(0xffffffffu, v, 0);
  sub = __shfl_sync(0xffffffffu, sub, 0);
  adm = __shfl_sync(0xffffffffu, adm, 0);
  quit = __shfl_sync(0xffffffffu, quit, 0);
  *subp = sub;
  // A launch that is winding down (quit) admits nothing: what it admitted it finishes, the
  // rest waits for the relaunch, so the launch never ends up serving on a few CTAs.
  if (sub != adm && quit == 0u) {
    int got = 0;
    if (lane == 0) got = atomicCAS(&c->admitted.v, adm, sub) == adm;
    if (!__shfl_sync(0xffffffffu, got, 0)) return kRetry;
    __threadfence();  // the records were copied before the count that published them
    *h = adm;
    *k = sub - adm;
    return kAdmit;
  }
  const uint8_t *order = short_only ? p.prio_short : p.prio;
  const int n = short_only ? (int)p.nshort : (int)p.nprio;
  // Two passes in priority order: first CTA-level work and thread-level queues whose backlog
  // fills a thread-per-instance claim (more than warp_max), then any non-empty queue.  A
  // device with work elsewhere lets a sponge stage's backlog build up into one claim of up
  // to 256 instances instead of spending a CTA slot on every few instances the stages before
  // it trickle in (a warp per instance holds a slot for 8 of them at about three times the
  // issue slots per permutation); an otherwise idle CTA takes what there is at once.
  for (int pass = 0; pass < 2; pass++) {
    for (int base = 0; base < n; base += 32) {
      const int j = base + lane;
      uint32_t hh = 0, tt = 0;
      int q = 0;
      bool ok = false;
      if (j < n) {
        q = order[j];
        hh = ld_relaxed(&c->head[q].v);
        tt = ld_relaxed(&c->tail[q].v);
        const int backlog = (int)(tt - hh);
        const int kind = kind_of(q_scheme(q), q_op(q), q_stage(q));
        ok = backlog > 0 && (pass == 1 || kind == K_CTA || (uint32_t)backlog > p.warp_max);
      }
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (!m) continue;
      const int src = __ffs(m) - 1;
      q = __shfl_sync(0xffffffffu, q, src);
      hh = __shfl_sync(0xffffffffu, hh, src);
      tt = __shfl_sync(0xffffffffu, tt, src);
      bool w;
      const uint32_t cap = cap_of(p, q, tt - hh, &w);
      const uint32_t n_take = min(tt - hh, cap);
      int got = 0;
      if (lane == 0) got = atomicCAS(&c->head[q].v, hh, hh + n_take) == hh;
      if (!__shfl_sync(0xffffffffu, got, 0)) return kRetry;
      *h = hh;
      *k = n_take;
      *warp = w;
      return q;
    }
  }
  return kNone;
}

// Thread 0 of an idle CTA: true when the launch should end (stop raised, another CTA gave
// up, or this one has been idle for idle_ns); otherwise sleeps until a push or a
// submission (at most about 40 microseconds) and returns false.  Only a CTA that sees every
// queue decides that the device is idle: a Saber-only CTA is idle whenever the work is
// all FrodoKEM.
__device__ bool idle(const Svc &p, bool short_only, uint64_t &idle_since, uint32_t version0, uint32_t sub0) {
  const uint64_t now = globaltimer_ns();
  if (idle_since == 0) idle_since = now;
  if (ld_relaxed(&p.ctl->stop.v) != 0u || ld_relaxed(&p.ctl->quit.v) != 0u) return true;
  if (!short_only && now - idle_since > p.idle_ns) {
    atomicExch(&p.ctl->quit.v, 1u);
    return true;
  }
  for (int i = 0; i < 64; i++) {
    if (ld_relaxed(&p.ctl->version.v) != version0 || ld_relaxed(&p.ctl->sub_tail.v) != sub0) break;
    __nanosleep(600);
  }
  return false;
}

__global__ void __launch_bounds__(256, 2) service_kernel(Svc p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint32_t s_q, s_h, s_k, s_w, s_ver, s_sub, s_exit, s_tmem;
  __shared__ uint32_t s_r[256];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid < 32) {
    tmem_alloc(&s_tmem, fdev::TC_TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = s_tmem;
  const bool short_only = blockIdx.x < p.short_ctas;
  uint64_t idle_since = 0;  // thread 0's
  while (true) {
    if (warp == 0) {
      uint32_t h = 0, k = 0, ver = 0, sub = 0;
      bool w = false;
      int q = kRetry, tries = 0;
      for (; tries < 64 && q == kRetry; tries++) {
        if (tries) __nanosleep(32u << min(tries, 6));  // another CTA took it: back off a little
        q = pick(p, short_only, &h, &k, &w, &ver, &sub);
      }
      if (lane == 0) {
        if (tries > 1) atomicAdd(p.stats + kQueues * 4 + 3, (unsigned long long)(tries - 1));
        s_q = q == kRetry ? kNone : q;  // lost every race: rescan after a short sleep
        s_h = h;
        s_k = k;
        s_w = w;
        s_ver = ver;
        s_sub = sub;
      }
    }
    __syncthreads();
    const int q = (int)s_q;
    const uint32_t h = s_h, k = s_k;
    const bool w = s_w != 0u;
    if (q == kNone) {
      if (tid == 0) {
        const uint64_t t0 = globaltimer_ns();
        s_exit = idle(p, short_only, idle_since, s_ver, s_sub) ? 1u : 0u;
        atomicAdd(p.stats + kQueues * 4, (unsigned long long)(globaltimer_ns() - t0));
      }
      __syncthreads();
      if (s_exit) break;
      continue;
    }
    if (tid == 0) idle_since = 0;
    if (q == kAdmit) {
      if (tid == 0) {
        atomicAdd(p.stats + kQueues * 4 + 1, 1ull);
        atomicAdd(p.stats + kQueues * 4 + 2, (unsigned long long)k);
      }
      for (uint32_t i = tid; i < k; i += blockDim.x) {
        const uint32_t r = (h + i) & p.qmask;
        push(p, queue_of(p.req[r].scheme, p.req[r].op, 0), r);
      }
      __syncthreads();
      if (tid == 0) wake(p);
      continue;
    }
    const int scheme = q_scheme(q), op = q_op(q), stage = q_stage(q);
    const int kind = kind_of(scheme, op, stage);
    const int code = code_of(scheme, op, stage, p.form);
    if ((uint32_t)tid < k) s_r[tid] = take(p, q, h + tid);
    __syncthreads();
    const uint64_t t_claim = tid == 0 ? globaltimer_ns() : 0;
    if (kind == K_CTA) {
      for (uint32_t i = 0; i < k; i++) {
        const uint32_t r = s_r[i];
        if (r != ~0u) cta_stage(code, p.req[r], smem, tbase, &p.ctl->err.v);
        __syncthreads();
        if (tid == 0 && r != ~0u) {
          const uint32_t e = ld_relaxed(&p.ctl->err.v);  // an expired wait inside the stage
          if (e != 0u) *p.host_err = e;
          advance(p, scheme, op, stage, r);
          wake(p);
        }
      }
    } else if (w) {
      const int slot = kind == K_THREAD2 ? warp >> 1 : warp, role = kind == K_THREAD2 ? warp & 1 : 0;
      if ((uint32_t)slot < k && s_r[slot] != ~0u) {  // warp-uniform: every lane runs the stage
        const uint32_t r = s_r[slot];
        warp_stage(p.key, code, p.req[r], role);
        // every lane's writes before the hand-off; host-visible after the last stage
        if (stage + 1 == nstages(scheme, op)) __threadfence_system();
        else __threadfence();
        __syncwarp();
        if (lane == 0) {
          if (kind == K_THREAD2) role_done(p, scheme, op, stage, r);
          else advance(p, scheme, op, stage, r);
          wake(p);
        }
      }
    } else {
      const int per = kind == K_THREAD2 ? 128 : 256;
      const int slot = tid % per, role = tid / per;
      if ((uint32_t)slot < k && s_r[slot] != ~0u) {
        const uint32_t r = s_r[slot];
        thread_stage(p.key, code, p.req[r], role);
        if (kind == K_THREAD2) role_done(p, scheme, op, stage, r);
        else advance(p, scheme, op, stage, r);
      }
    }
    __syncthreads();  // s_r and the claim words are rewritten by the next pick
    if (tid == 0) {
      if (kind != K_CTA && !w) wake(p);  // the thread-per-instance claim's pushes
      unsigned long long *qs = p.stats + q * 4;
      atomicAdd(qs, 1ull);
      atomicAdd(qs + 1, (unsigned long long)k);
      if (w) atomicAdd(qs + 2, 1ull);
      atomicAdd(qs + 3, (unsigned long long)(globaltimer_ns() - t_claim));
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid < 32) {
    tc_fence_after();
    tmem_dealloc(tbase, fdev::TC_TMEM_COLS);
  }
}

// Fresh queues: entry k of every queue carries sequence k (free for lap 0).
__global__ void init_entries_kernel(unsigned long long *ent, uint32_t slots) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < (size_t)kQueues * slots) ent[i] = (unsigned long long)(i % slots) << 32;
}


// ---------------------------------------------------------------- host
constexpr int kWords = 256;  // pinned words carrying published counts (one per submission)

uint32_t rec_bytes(int scheme) { return (uint32_t)(scheme <= 1 ? kFrodoRec : saber_rec_bytes(scheme)); }

// Queue priorities: Saber before FrodoKEM (a sub-millisecond chain next to a multi-millisecond
// one), and within each the later stages first, so requests already in flight finish before
// new ones start.  Short-only CTAs see the Saber queues alone.
void build_priorities(Svc &p) {
  std::vector<int> qs;
  for (int scheme = 0; scheme < 5; scheme++)
    for (int op = 0; op < 3; op++)
      for (int st = 0; st < nstages(scheme, op); st++) qs.push_back(queue_of(scheme, op, st));
  auto key = [](int q) {
    const int scheme = q_scheme(q), op = q_op(q), st = q_stage(q);
    return std::make_tuple(scheme <= 1 ? 1 : 0, nstages(scheme, op) - 1 - st, scheme, op);
  };
  std::stable_sort(qs.begin(), qs.end(), [&](int a, int b) { return key(a) < key(b); });
  p.nprio = p.nshort = 0;
  for (int q : qs) {
    p.prio[p.nprio++] = (uint8_t)q;
    if (q_scheme(q) >= 2) p.prio_short[p.nshort++] = (uint8_t)q;
  }
}

cudaError_t launch(const Svc &p, int grid, cudaStream_t st) {
  service_kernel<<<grid, 256, kSmem, st>>>(p);
  return cudaGetLastError();
}

}  // namespace
}  // namespace serve
}  // namespace dpkem

using namespace dpkem;
using namespace dpkem::abi;

struct dpkem_service {
  dpkem_ctx *c = nullptr;
  int form = 0;
  bool has_key = false;
  cudaStream_t kst = nullptr, cst = nullptr;  // the kernel's stream; the submissions' copy stream
  cudaEvent_t kev = nullptr;                  // recorded after each launch
  cudaEvent_t wev[serve::kWords] = {};
  bool running = false;
  int grid = 0;
  uint32_t slots = 0;
  serve::Svc p{};
  uint8_t *dmem = nullptr;
  serve::Ctl *ctl = nullptr;
  mixed::DevReq *d_req = nullptr;
  uint8_t *d_scr = nullptr;
  uint64_t scr_bytes = 0;
  mixed::DevReq *h_req = nullptr;  // pinned mirror of d_req (the copies' source)
  uint32_t *h_words = nullptr;     // pinned published counts
  uint32_t *h_map = nullptr;       // host-mapped: [slots] completion words, then the error word
  uint64_t next = 0, oldest = 0, nsubmit = 0, launches = 0, scanned = 0;
  uint64_t scr_head = 0, scr_tail = 0;
  std::vector<uint64_t> scr_end;   // per slot: end of its scratch record (monotone offsets)
  std::vector<uint8_t> complete;   // per slot: completion seen, slot not yet released
  std::vector<uint64_t> report;    // completed tickets not yet returned by poll
  size_t report_head = 0;
  std::mutex mu;
};

namespace {

// Completions since the last scan: queued for poll, and slots released in ticket order.
void scan(dpkem_service *s) {
  const uint32_t mask = s->slots - 1;
  volatile const uint32_t *hd = s->h_map;
  for (uint64_t t = std::max(s->scanned, s->oldest); t < s->next; t++) {
    const uint32_t r = (uint32_t)t & mask;
    if (!s->complete[r] && hd[r] == (uint32_t)(t + 1)) {
      s->complete[r] = 1;
      s->report.push_back(t);
    }
  }
  while (s->oldest < s->next && s->complete[(uint32_t)s->oldest & mask]) {
    const uint32_t r = (uint32_t)s->oldest & mask;
    s->complete[r] = 0;
    s->scr_tail = s->scr_end[r];
    s->oldest++;
  }
  s->scanned = s->oldest;
  if (s->report_head > 4096 && s->report_head * 2 > s->report.size()) {
    s->report.erase(s->report.begin(), s->report.begin() + (ptrdiff_t)s->report_head);
    s->report_head = 0;
  }
}

// Relaunch the kernel when it has ended (idle limit) while requests are outstanding.
int ensure_running(dpkem_service *s) {
  if (s->running) {
    const cudaError_t q = cudaEventQuery(s->kev);
    if (q == cudaSuccess) s->running = false;
    else if (q != cudaErrorNotReady) return cuda_status(q);
  }
  if (s->running || s->oldest == s->next) return DPKEM_OK;
  cudaError_t e = cudaMemsetAsync(&s->ctl->quit.v, 0, 4, s->kst);
  if (e == cudaSuccess) e = serve::launch(s->p, s->grid, s->kst);
  if (e == cudaSuccess) e = cudaEventRecord(s->kev, s->kst);
  if (e != cudaSuccess) return cuda_status(e);
  s->running = true;
  s->launches++;
  return DPKEM_OK;
}

// Copies pinned word w (holding v) to a control word on the copy stream.
cudaError_t publish(dpkem_service *s, uint32_t *dst, uint32_t v) {
  const int w = (int)(s->nsubmit++ % serve::kWords);
  cudaError_t e = cudaEventSynchronize(s->wev[w]);  // its previous copy has run
  if (e != cudaSuccess) return e;
  s->h_words[w] = v;
  e = cudaMemcpyAsync(dst, &s->h_words[w], 4, cudaMemcpyHostToDevice, s->cst);
  if (e == cudaSuccess) e = cudaEventRecord(s->wev[w], s->cst);
  return e;
}

void release(dpkem_service *s) {
  if (s->kst) cudaStreamSynchronize(s->kst);
  if (s->cst) cudaStreamSynchronize(s->cst);
  for (cudaEvent_t &ev : s->wev)
    if (ev) cudaEventDestroy(ev);
  if (s->kev) cudaEventDestroy(s->kev);
  if (s->kst) cudaStreamDestroy(s->kst);
  if (s->cst) cudaStreamDestroy(s->cst);
  if (s->dmem) cudaFree(s->dmem);
  if (s->h_req) cudaFreeHost(s->h_req);
  if (s->h_words) cudaFreeHost(s->h_words);
  if (s->h_map) cudaFreeHost(s->h_map);
  cudaGetLastError();
  delete s;
}

}  // namespace

int dpkem_service_default_config(dpkem_service_config *cfg) {
  if (!cfg) return set_status(DPKEM_EINVAL);
  *cfg = dpkem_service_config{};
  cfg->max_inflight = 16384;
  cfg->idle_ms = 1000;
  cfg->saber_ctas = 0;
  cfg->warp_max = 32;
  cfg->scratch_bytes = 0;
  cfg->coin_key = nullptr;
  return set_status(DPKEM_OK);
}

int dpkem_service_open(dpkem_ctx *c, int form, const dpkem_service_config *cfg_in, dpkem_service **out) {
  if (!c || !out) return set_status(DPKEM_EINVAL);
  *out = nullptr;
  if (form != DPKEM_FORM_DP4A && form != DPKEM_FORM_TC && form != DPKEM_FORM_INT32) return set_status(DPKEM_EINVAL);
  dpkem_service_config cfg;
  dpkem_service_default_config(&cfg);
  if (cfg_in) cfg = *cfg_in;
  if (cfg.max_inflight == 0 || cfg.max_inflight > (1u << 20) || cfg.idle_ms == 0 || cfg.idle_ms > 600000)
    return set_status(DPKEM_EINVAL);
  uint32_t slots = 64;
  while (slots < cfg.max_inflight) slots <<= 1;
  const uint64_t scr = cfg.scratch_bytes ? cfg.scratch_bytes : (uint64_t)slots * mixed::kFrodoRec;
  if (scr < mixed::kFrodoRec) return set_status(DPKEM_EINVAL);
  const size_t o_stats = up(sizeof(serve::Ctl)), o_req = o_stats + up(serve::kStats * 8), o_done = o_req + up((size_t)slots * sizeof(mixed::DevReq));
  const size_t o_ent = o_done + up((size_t)slots * 4), o_scr = o_ent + up((size_t)serve::kQueues * slots * 8);
  const size_t total = o_scr + up(scr);
  if (total > c->budget) return set_status(DPKEM_ENOMEM);
  std::lock_guard<std::mutex> lock(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) return set_status(cuda_status(cudaErrorInvalidDevice));
  dpkem_service *s = new dpkem_service();
  s->c = c;
  s->form = form;
  s->slots = slots;
  s->scr_bytes = scr;
  s->has_key = cfg.coin_key != nullptr;
  s->scr_end.assign(slots, 0);
  s->complete.assign(slots, 0);
  cudaError_t e = cudaStreamCreateWithFlags(&s->kst, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->cst, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->kev, cudaEventDisableTiming);
  for (int w = 0; w < serve::kWords && e == cudaSuccess; w++)
    e = cudaEventCreateWithFlags(&s->wev[w], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&s->dmem, total);
  if (e == cudaSuccess) e = cudaHostAlloc(&s->h_req, (size_t)slots * sizeof(mixed::DevReq), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc(&s->h_words, serve::kWords * 4, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc(&s->h_map, ((size_t)slots + 32) * 4, cudaHostAllocMapped);
  uint32_t *d_map = nullptr;
  if (e == cudaSuccess) e = cudaHostGetDevicePointer(&d_map, s->h_map, 0);
  if (e == cudaSuccess) {
    std::memset(s->h_map, 0, ((size_t)slots + 32) * 4);
    s->ctl = reinterpret_cast<serve::Ctl *>(s->dmem);
    s->d_req = reinterpret_cast<mixed::DevReq *>(s->dmem + o_req);
    s->d_scr = s->dmem + o_scr;
    e = cudaMemsetAsync(s->dmem, 0, o_ent, s->kst);  // control words, records, role counters
  }
  unsigned long long *ent = e == cudaSuccess ? reinterpret_cast<unsigned long long *>(s->dmem + o_ent) : nullptr;
  if (e == cudaSuccess) {
    const size_t n = (size_t)serve::kQueues * slots;
    serve::init_entries_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->kst>>>(ent, slots);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaFuncSetAttribute(serve::service_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 mixed::kSmem);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->kst);
  if (e == cudaSuccess) {
    int sms = 0, occ = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, serve::service_kernel, 256, mixed::kSmem);
    s->grid = std::max(1, sms * std::max(1, std::min(occ, 2)));
    if (c->max_ctas > 0) s->grid = std::min(s->grid, c->max_ctas);
  }
  if (e != cudaSuccess) {
    const int rc = cuda_status(e);
    release(s);
    return set_status(rc);
  }
  serve::Svc &p = s->p;
  p.ctl = s->ctl;
  p.stats = reinterpret_cast<unsigned long long *>(s->dmem + o_stats);
  p.req = s->d_req;
  p.done = reinterpret_cast<uint32_t *>(s->dmem + o_done);
  p.ent = ent;
  p.qmask = slots - 1;
  p.short_ctas = std::min<uint32_t>(cfg.saber_ctas, (uint32_t)std::max(0, s->grid - 1));
  p.warp_max = cfg.warp_max;
  p.form = form;
  serve::build_priorities(p);
  p.idle_ns = (uint64_t)cfg.idle_ms * 1000000ull;
  p.host_done = d_map;
  p.host_err = d_map + slots;
  p.key = default_coin_key();
  if (cfg.coin_key)
    for (int q = 0; q < 4; q++) {
      uint32_t lo, hi;
      std::memcpy(&lo, cfg.coin_key + 8 * q, 4);
      std::memcpy(&hi, cfg.coin_key + 8 * q + 4, 4);
      p.key.w[q] = make_uint2(lo, hi);
    }
  *out = s;
  return set_status(DPKEM_OK);
}

int dpkem_service_submit(dpkem_service *s, size_t n, const dpkem_request *reqs, size_t *accepted,
                         uint64_t *first_ticket) {
  if (accepted) *accepted = 0;
  if (!s) return set_status(DPKEM_EINVAL);
  if (n == 0) return set_status(DPKEM_OK);
  int rc = check_requests(n, reqs, s->has_key);
  if (rc) return set_status(rc);
  std::lock_guard<std::mutex> lock(s->mu);
  cudaSetDevice(s->c->device);
  scan(s);
  const uint32_t mask = s->slots - 1;
  const uint64_t first = s->next;
  size_t acc = 0;
  // Admission: a request is taken while a slot is free and the live scratch (from the oldest
  // incomplete request's record to the newest) leaves room for its record.
  for (; acc < n; acc++) {
    const dpkem_request &r = reqs[acc];
    if (s->next - s->oldest >= s->slots) break;
    const uint64_t need = serve::rec_bytes(r.scheme);
    uint64_t pos = s->scr_head;
    if (pos % s->scr_bytes + need > s->scr_bytes) pos += s->scr_bytes - pos % s->scr_bytes;  // no record wraps
    if (pos + need - s->scr_tail > s->scr_bytes) break;
    const uint32_t slot = (uint32_t)s->next & mask;
    uint8_t *rec = s->d_scr + pos % s->scr_bytes;
    mixed::DevReq d{r.scheme, r.op, r.in0, r.in1, r.out0, r.out1, rec, s->next, 0u, (uint32_t)s->next};
    if (s->has_key && !r.in0 && r.op != OP_DEC) {  // coins drawn on the device into the record
      d.in0 = rec + (r.scheme <= 1 ? mixed::kFrodoCoins : mixed::saber_coins_off(r.scheme));
      d.gen = 1;
    }
    s->h_req[slot] = d;
    s->scr_end[slot] = pos + need;
    s->scr_head = pos + need;
    s->complete[slot] = 0;
    s->h_map[slot] = 0;
    s->next++;
  }
  if (accepted) *accepted = acc;
  if (first_ticket) *first_ticket = first;
  if (acc == 0) return set_status(DPKEM_EAGAIN);
  // records (one or two contiguous slot ranges), then the published count, on one stream
  const uint32_t a = (uint32_t)first & mask;
  const size_t run = std::min<size_t>(acc, s->slots - a);
  cudaError_t e = cudaMemcpyAsync(s->d_req + a, s->h_req + a, run * sizeof(mixed::DevReq), cudaMemcpyHostToDevice,
                                  s->cst);
  if (e == cudaSuccess && run < acc)
    e = cudaMemcpyAsync(s->d_req, s->h_req, (acc - run) * sizeof(mixed::DevReq), cudaMemcpyHostToDevice, s->cst);
  if (e == cudaSuccess) e = publish(s, &s->ctl->sub_tail.v, (uint32_t)s->next);
  if (e != cudaSuccess) return set_status(cuda_status(e));
  return set_status(ensure_running(s));
}

int dpkem_service_poll(dpkem_service *s, uint64_t *tickets, size_t max, size_t *n_done) {
  if (n_done) *n_done = 0;
  if (!s || (max && !tickets)) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(s->mu);
  cudaSetDevice(s->c->device);
  scan(s);
  size_t k = 0;
  while (k < max && s->report_head < s->report.size()) tickets[k++] = s->report[s->report_head++];
  if (n_done) *n_done = k;
  const int rc = ensure_running(s);
  if (rc) return set_status(rc);
  return set_status(s->h_map[s->slots] ? DPKEM_ETIMEOUT : DPKEM_OK);
}

int dpkem_service_drain(dpkem_service *s, uint32_t timeout_ms) {
  if (!s) return set_status(DPKEM_EINVAL);
  const auto t0 = std::chrono::steady_clock::now();
  while (true) {
    {
      std::lock_guard<std::mutex> lock(s->mu);
      cudaSetDevice(s->c->device);
      scan(s);
      const int rc = ensure_running(s);
      if (rc) return set_status(rc);
      if (s->h_map[s->slots]) return set_status(DPKEM_ETIMEOUT);
      if (s->oldest == s->next) return set_status(DPKEM_OK);
    }
    if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms))
      return set_status(DPKEM_ETIMEOUT);
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

int dpkem_service_stats(dpkem_service *s, uint64_t *submitted, uint64_t *completed, uint64_t *launches,
                        int *running) {
  if (!s) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(s->mu);
  cudaSetDevice(s->c->device);
  scan(s);
  if (s->running && cudaEventQuery(s->kev) == cudaSuccess) s->running = false;
  cudaGetLastError();
  if (submitted) *submitted = s->next;
  if (completed) *completed = s->oldest;
  if (launches) *launches = s->launches;
  if (running) *running = s->running ? 1 : 0;
  return set_status(DPKEM_OK);
}

int dpkem_service_counters(dpkem_service *s, uint64_t *out, size_t n, int reset) {
  if (!s || (n && !out)) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(s->mu);
  cudaSetDevice(s->c->device);
  const size_t k = std::min<size_t>(n, serve::kStats);
  cudaError_t e = cudaSuccess;
  if (k) e = cudaMemcpyAsync(out, s->p.stats, k * 8, cudaMemcpyDeviceToHost, s->cst);
  if (e == cudaSuccess && reset) e = cudaMemsetAsync(s->p.stats, 0, serve::kStats * 8, s->cst);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->cst);
  return set_status(cuda_status(e));
}

int dpkem_service_close(dpkem_service *s) {
  if (!s) return set_status(DPKEM_EINVAL);
  cudaSetDevice(s->c->device);
  int rc = dpkem_service_drain(s, 30000);
  {
    std::lock_guard<std::mutex> lock(s->mu);
    cudaError_t e = publish(s, &s->ctl->stop.v, 1u);
    // the launch ends once idle; its idle limit bounds the wait even if stop were missed
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->cst);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->kst);
    if (e != cudaSuccess && rc == DPKEM_OK) rc = cuda_status(e);
    if (rc == DPKEM_OK && s->h_map[s->slots]) rc = DPKEM_ETIMEOUT;
  }
  release(s);
  return set_status(rc);
}
