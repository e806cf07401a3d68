// Wire-format entry points (include/dpkem_wire.h): request/response frames, the
// frame runner on the GPU, host registration, and the shared-memory ring protocol.
//
// dpkem_frames_run moves a block of request frames to the device as it is (one copy per
// pipeline chunk), points the persistent mixed-batch kernel's request table straight at
// the payloads inside the device copy, writes the response frames next to them (payloads
// by the mixed kernel, headers by frame_headers_kernel) and copies each chunk's response
// range back in one piece.  No per-frame copies on either side.
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <utility>
#include <vector>

#include "../../include/dpkem.h"
#include "../../include/dpkem_wire.h"
#include "common.cuh"
#include "ctx.h"

using namespace dpkem;
using namespace dpkem::abi;

namespace {

constexpr size_t kHdr = DPKEM_FRAME_HEADER;
constexpr size_t kGroupMin = 256;  // smallest pipeline chunk, in frames

size_t pad16(size_t x) { return (x + 15) & ~(size_t)15; }
size_t pad32(size_t x) { return (x + 31) & ~(size_t)31; }

// Offsets of the payload sections inside a frame (0 = section absent) and frame sizes.
struct Layout {
  size_t req, resp;
  size_t in0, in1, out0, out1;
  size_t resp_end;  // end of the last response section (zero padding follows)
};

bool layout_of(int scheme, int op, Layout *L) {
  Sizes z;
  if (!scheme_sizes(scheme, &z)) return false;
  switch (op) {
    case DPKEM_OP_KEYPAIR:
      *L = {pad32(kHdr + pad16(z.kpc)), pad32(kHdr + z.pk + z.sk), kHdr, 0, kHdr, kHdr + z.pk, kHdr + z.pk + z.sk};
      return true;
    case DPKEM_OP_ENC:
      *L = {pad32(kHdr + pad16(z.encc) + z.pk), pad32(kHdr + z.ct + pad16(z.ss)), kHdr, kHdr + pad16(z.encc), kHdr,
            kHdr + z.ct, kHdr + z.ct + z.ss};
      return true;
    case DPKEM_OP_DEC:
      *L = {pad32(kHdr + z.ct + z.sk), pad32(kHdr + pad16(z.ss)), kHdr, kHdr + z.ct, kHdr, 0, kHdr + z.ss};
      return true;
    default:
      return false;
  }
}

struct Frame {
  int scheme, op;
  size_t off, resp_off;  // frame offset in the request block, its response's in the response block
};

struct ScanResult {
  size_t frames = 0, used = 0, resp_bytes = 0;
};

// Parses a block of request frames (see dpkem_frames_scan); `out` may be null.
int scan(const uint8_t *req, size_t bytes, size_t max_frames, std::vector<Frame> *out, ScanResult *r) {
  size_t pos = 0, count = 0, rtot = 0;
  while (pos < bytes && (max_frames == 0 || count < max_frames)) {
    if (bytes - pos < kHdr) return DPKEM_EINVAL;
    dpkem_frame_header h;
    std::memcpy(&h, req + pos, sizeof(h));
    if (h.magic == DPKEM_FRAME_PAD) {
      if (h.frame_bytes < kHdr || h.frame_bytes % DPKEM_FRAME_ALIGN || h.frame_bytes > bytes - pos)
        return DPKEM_EINVAL;
      pos += h.frame_bytes;
      continue;
    }
    Layout L;
    if (h.magic != DPKEM_FRAME_MAGIC || h.version != DPKEM_FRAME_VERSION || !layout_of(h.scheme, h.op, &L) ||
        h.frame_bytes != L.req || L.req > bytes - pos)
      return DPKEM_EINVAL;
    if (out) out->push_back(Frame{h.scheme, h.op, pos, rtot});
    rtot += L.resp;
    pos += L.req;
    count++;
  }
  *r = ScanResult{count, pos, rtot};
  return DPKEM_OK;
}

// Response frame sizes and payload ends indexed by scheme * 3 + op (0 for unknown schemes).
void resp_table(uint32_t bytes[15], uint32_t end[15]) {
  for (int s = 0; s < 5; s++)
    for (int op = 0; op < 3; op++) {
      Layout L;
      const bool ok = layout_of(s, op, &L);
      bytes[s * 3 + op] = ok ? (uint32_t)L.resp : 0u;
      end[s * 3 + op] = ok ? (uint32_t)L.resp_end : 0u;
    }
}

// One pipeline chunk: frames [a, b) of the block.
struct Group {
  size_t a, b;
  size_t req_start, req_len, resp_start, resp_len;
  size_t need;  // device bytes: request copy + response copy + mixed plan
};

std::vector<mixed::Req> group_reqs(const std::vector<Frame> &fr, const Group &g, uint8_t *d_req, uint8_t *d_resp) {
  std::vector<mixed::Req> rq(g.b - g.a);
  for (size_t i = g.a; i < g.b; i++) {
    const Frame &f = fr[i];
    Layout L;
    layout_of(f.scheme, f.op, &L);
    uint8_t *in = d_req + (f.off - g.req_start);
    uint8_t *out = d_resp + (f.resp_off - g.resp_start);
    rq[i - g.a] = mixed::Req{f.scheme, f.op, in + L.in0, L.in1 ? in + L.in1 : nullptr, out + L.out0,
                             L.out1 ? out + L.out1 : nullptr};
  }
  return rq;
}

std::vector<Group> make_groups(const std::vector<Frame> &fr, size_t per) {
  std::vector<Group> gs;
  for (size_t a = 0; a < fr.size(); a += per) {
    const size_t b = std::min(fr.size(), a + per);
    Layout Lb;
    layout_of(fr[b - 1].scheme, fr[b - 1].op, &Lb);
    Group g{a, b, fr[a].off, fr[b - 1].off + Lb.req - fr[a].off, fr[a].resp_off,
            fr[b - 1].resp_off + Lb.resp - fr[a].resp_off, 0};
    // plan bytes depend only on the (scheme, op) mix, so placeholder pointers will do
    const std::vector<mixed::Req> rq = group_reqs(fr, g, nullptr, nullptr);
    g.need = up(g.req_len) + up(g.resp_len) + up(mixed::plan_bytes(rq.data(), rq.size(), nullptr));
    gs.push_back(g);
  }
  return gs;
}

dpkem_ring_control *ring_ctl(void *base) {
  auto *c = static_cast<dpkem_ring_control *>(base);
  if (!c || c->magic != DPKEM_RING_MAGIC || c->capacity == 0 || c->capacity % 4096) return nullptr;
  return c;
}
uint8_t *ring_req(void *base) { return static_cast<uint8_t *>(base) + DPKEM_RING_CONTROL; }
uint8_t *ring_resp(void *base, size_t cap) { return static_cast<uint8_t *>(base) + DPKEM_RING_CONTROL + cap; }
uint64_t ld_acq(const uint64_t *p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }
void st_rel(uint64_t *p, uint64_t v) { __atomic_store_n(p, v, __ATOMIC_RELEASE); }

void write_pad(uint8_t *at, size_t bytes) {
  dpkem_frame_header h{};
  h.magic = DPKEM_FRAME_PAD;
  h.version = DPKEM_FRAME_VERSION;
  h.frame_bytes = (uint32_t)bytes;
  std::memcpy(at, &h, sizeof(h));
}

// Enqueues a frame block on the context's streams (see dpkem_frames_run); frames_finish
// waits for it.  *resp_bytes is set on success.
int frames_submit(dpkem_ctx *c, int form, const uint8_t *req, size_t req_bytes, uint8_t *resp, size_t resp_cap,
                  size_t *resp_bytes) {
  if (!c || !resp_bytes || (!req && req_bytes)) return DPKEM_EINVAL;
  if (form != DPKEM_FORM_DP4A && form != DPKEM_FORM_TC && form != DPKEM_FORM_INT32) return DPKEM_EINVAL;
  *resp_bytes = 0;
  std::vector<Frame> fr;
  ScanResult sr;
  int rc = scan(req, req_bytes, 0, &fr, &sr);
  if (rc) return rc;
  if (sr.resp_bytes > resp_cap || (!resp && sr.resp_bytes)) return DPKEM_EINVAL;
  if (fr.empty()) return DPKEM_OK;

  std::lock_guard<std::mutex> lock(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) return cuda_status(cudaErrorInvalidDevice);
  // Chunks: up to pipe_chunks of at least kGroupMin frames, all in flight on their own
  // streams; halved until the chunks in flight fit the context's budget.
  const size_t n = fr.size();
  int npipe = (int)std::min<size_t>(std::min(std::max(tuning().pipe_chunks, 1), kPipeChunks),
                                    std::max<size_t>(1, n / kGroupMin));
  size_t per = (n + npipe - 1) / npipe;
  std::vector<Group> gs;
  size_t region = 0;
  while (true) {
    gs = make_groups(fr, per);
    region = 0;
    for (const Group &g : gs) region = std::max(region, g.need);
    npipe = (int)std::min<size_t>(npipe, gs.size());
    if (region * npipe <= c->budget) break;
    if (npipe > 1) {
      npipe--;
      continue;
    }
    if (per == 1) return DPKEM_ENOMEM;
    per = (per + 1) / 2;
  }
  if ((rc = ensure_arena(c, region * npipe)) != DPKEM_OK) return rc;

  cudaStream_t st = c->stream;
  cudaError_t e = cudaStreamWaitEvent(st, c->last, 0);
  if (e == cudaSuccess) e = cudaEventRecord(c->pev[0], st);
  for (int j = 0; j < npipe && e == cudaSuccess; j++) e = cudaStreamWaitEvent(c->pipe[j], c->pev[0], 0);
  int grid = 0;
  if (e == cudaSuccess) e = persistent_grid(c, &grid);
  uint32_t rtab[15], rend[15];
  resp_table(rtab, rend);
  std::vector<std::vector<uint8_t>> plans(gs.size(), std::vector<uint8_t>(mixed::plan_struct_bytes()));
  for (size_t k = 0; k < gs.size() && e == cudaSuccess; k++) {
    const Group &g = gs[k];
    cudaStream_t sj = c->pipe[k % npipe];
    uint8_t *d_req = c->arena + (k % npipe) * region;
    uint8_t *d_resp = d_req + up(g.req_len);
    uint8_t *d_plan = d_resp + up(g.resp_len);
    const std::vector<mixed::Req> rq = group_reqs(fr, g, d_req, d_resp);
    const int sj_idx = (int)(k % npipe);
    uint8_t *stage = stage_for(c, sj_idx, mixed::plan_table_bytes(rq.data(), rq.size()));
    e = cudaMemcpyAsync(d_req, req + g.req_start, g.req_len, cudaMemcpyHostToDevice, sj);
    if (e == cudaSuccess)
      e = mixed::plan_build(rq.data(), rq.size(), form, grid, d_plan, region - (size_t)(d_plan - d_req), c->d_err, sj,
                            plans[k].data(), nullptr, 0, stage, stage ? c->h_stage_bytes[sj_idx] : 0);
    if (e == cudaSuccess && stage) stage_used(c, sj_idx, sj);
    if (e == cudaSuccess) e = mixed::plan_launch(plans[k].data(), rq.size(), grid, sj);
    if (e == cudaSuccess) e = mixed::frame_headers_launch(plans[k].data(), rq.size(), rtab, rend, sj);
    if (e == cudaSuccess) e = cudaMemcpyAsync(resp + g.resp_start, d_resp, g.resp_len, cudaMemcpyDeviceToHost, sj);
  }
  for (int j = 0; j < npipe && e == cudaSuccess; j++) {
    e = cudaEventRecord(c->pev[j], c->pipe[j]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, c->pev[j], 0);
  }
  if (e == cudaSuccess) e = cudaEventRecord(c->last, st);
  if (e != cudaSuccess) return cuda_status(e);
  *resp_bytes = sr.resp_bytes;
  return DPKEM_OK;
}

// Waits for the context's last submitted block; reports (and clears) a device timeout.
int frames_finish(dpkem_ctx *c) {
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  uint32_t err = 0;
  cudaError_t e = cudaEventSynchronize(c->last);
  if (e == cudaSuccess) e = cudaMemcpy(&err, c->d_err, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e);
  if (err) {
    cudaMemset(c->d_err, 0, 4);
    return DPKEM_ETIMEOUT;
  }
  return DPKEM_OK;
}

bool frames_done(dpkem_ctx *c) { return cudaEventQuery(c->last) != cudaErrorNotReady; }

// Server-side position in a ring: where the next batch starts, plus PAD bytes passed over
// that no published batch has accounted for yet.
struct Cursor {
  uint64_t req, resp;
  uint64_t req_pending, resp_pending;
};

struct RingBatch {
  size_t req_off, req_bytes, req_advance, resp_off, resp_bytes, resp_advance, n;
};

void publish(dpkem_ring_control *c, uint64_t req_advance, uint64_t resp_advance, uint64_t n) {
  st_rel(&c->resp_tail, c->resp_tail + resp_advance);  // responses first, then free the requests
  st_rel(&c->req_head, c->req_head + req_advance);
  if (n) st_rel(&c->served, c->served + n);
}

// Takes up to max_frames contiguous request frames at cur->req and reserves response room
// at cur->resp; advances the cursor.  EAGAIN with nothing taken may still have moved the
// cursor over PAD frames (recorded in the pending counts).
int acquire_at(void *base, size_t max_frames, Cursor *cur, RingBatch *out) {
  dpkem_ring_control *c = ring_ctl(base);
  const uint64_t cap = c->capacity, tail = ld_acq(&c->req_tail);
  const uint8_t *ring = ring_req(base);
  while (cur->req < tail) {  // skip PAD frames
    dpkem_frame_header h;
    std::memcpy(&h, ring + cur->req % cap, sizeof(h));
    if (h.magic != DPKEM_FRAME_PAD) break;
    if (h.frame_bytes < kHdr || h.frame_bytes % DPKEM_FRAME_ALIGN) return DPKEM_EINVAL;
    cur->req += h.frame_bytes;
    cur->req_pending += h.frame_bytes;
  }
  if (cur->req == tail) return DPKEM_EAGAIN;
  const uint64_t pos = cur->req % cap, avail = std::min<uint64_t>(tail - cur->req, cap - pos);
  // response room: contiguous at the cursor, or from 0 after a PAD to the end
  const uint64_t rfree = cap - (cur->resp - ld_acq(&c->resp_head)), rpos = cur->resp % cap;
  size_t k = 0, used = 0, rneed = 0;
  bool wrap = false;
  while (used < avail && (max_frames == 0 || k < max_frames)) {
    dpkem_frame_header h;
    std::memcpy(&h, ring + pos + used, sizeof(h));
    if (h.magic == DPKEM_FRAME_PAD) break;  // a PAD ends the contiguous run
    Layout L;
    if (h.magic != DPKEM_FRAME_MAGIC || h.version != DPKEM_FRAME_VERSION || !layout_of(h.scheme, h.op, &L) ||
        h.frame_bytes != L.req || L.req > avail - used)
      return DPKEM_EINVAL;
    if (L.resp > cap) return DPKEM_EINVAL;  // a response that can never fit
    const uint64_t r = rneed + L.resp;
    const bool fits_here = rpos + r <= cap && r <= rfree;
    const bool fits_wrapped = rpos != 0 && (cap - rpos) + r <= rfree;
    if (!fits_here && !fits_wrapped) break;
    wrap = !fits_here;
    rneed = r;
    used += L.req;
    k++;
  }
  if (k == 0) {
    // The first response fits neither before the end nor after a PAD: close the end with
    // a PAD now (if it fits), so the response starts at 0 once the client has caught up.
    if (rpos != 0 && cap - rpos <= rfree) {
      write_pad(ring_resp(base, cap) + rpos, cap - rpos);
      cur->resp += cap - rpos;
      cur->resp_pending += cap - rpos;
    }
    return DPKEM_EAGAIN;
  }
  uint64_t rpad = 0;
  if (wrap) {
    write_pad(ring_resp(base, cap) + rpos, cap - rpos);
    rpad = cap - rpos;
  }
  *out = RingBatch{pos, used, (size_t)(cur->req_pending + used), wrap ? 0 : rpos, rneed,
                   (size_t)(cur->resp_pending + rpad + rneed), k};
  cur->req += used;
  cur->resp += rpad + rneed;
  cur->req_pending = cur->resp_pending = 0;
  return DPKEM_OK;
}

}  // namespace

extern "C" {

int dpkem_frame_bytes(int scheme, int op, size_t *request_bytes, size_t *response_bytes) {
  Layout L;
  if (!layout_of(scheme, op, &L)) return set_status(DPKEM_EINVAL);
  if (request_bytes) *request_bytes = L.req;
  if (response_bytes) *response_bytes = L.resp;
  return set_status(DPKEM_OK);
}

int dpkem_frames_scan(const uint8_t *req, size_t req_bytes, size_t max_frames, size_t *n_frames, size_t *used_bytes,
                      size_t *response_bytes) {
  if (!req && req_bytes) return set_status(DPKEM_EINVAL);
  ScanResult r;
  const int rc = scan(req, req_bytes, max_frames, nullptr, &r);
  if (rc) return set_status(rc);
  if (n_frames) *n_frames = r.frames;
  if (used_bytes) *used_bytes = r.used;
  if (response_bytes) *response_bytes = r.resp_bytes;
  return set_status(DPKEM_OK);
}

int dpkem_frames_run(dpkem_ctx *c, int form, const uint8_t *req, size_t req_bytes, uint8_t *resp, size_t resp_cap,
                     size_t *resp_bytes) {
  int rc = frames_submit(c, form, req, req_bytes, resp, resp_cap, resp_bytes);
  if (rc) return set_status(rc);
  rc = frames_finish(c);
  if (rc) *resp_bytes = 0;
  return set_status(rc);
}

int dpkem_host_register(void *ptr, size_t bytes) {
  if (!ptr || !bytes) return set_status(DPKEM_EINVAL);
  return set_status(cuda_status(cudaHostRegister(ptr, bytes, cudaHostRegisterPortable)));
}

int dpkem_host_unregister(void *ptr) {
  if (!ptr) return set_status(DPKEM_EINVAL);
  return set_status(cuda_status(cudaHostUnregister(ptr)));
}

// ---------------------------------------------------------------- shared-memory ring
size_t dpkem_ring_bytes(size_t capacity) { return DPKEM_RING_CONTROL + 2 * capacity; }

int dpkem_ring_init(void *base, size_t capacity) {
  if (!base || capacity == 0 || capacity % 4096) return set_status(DPKEM_EINVAL);
  std::memset(base, 0, DPKEM_RING_CONTROL);
  auto *c = static_cast<dpkem_ring_control *>(base);
  c->version = 1;
  c->capacity = capacity;
  __atomic_store_n(&c->magic, DPKEM_RING_MAGIC, __ATOMIC_RELEASE);
  return set_status(DPKEM_OK);
}

int dpkem_ring_push(void *base, const uint8_t *frames, size_t bytes, size_t *pushed) {
  dpkem_ring_control *c = ring_ctl(base);
  if (!c || !pushed || (!frames && bytes)) return set_status(DPKEM_EINVAL);
  *pushed = 0;
  std::vector<Frame> fr;
  ScanResult sr;
  int rc = scan(frames, bytes, 0, &fr, &sr);
  if (rc) return set_status(rc);
  const uint64_t cap = c->capacity, tail = c->req_tail, free = cap - (tail - ld_acq(&c->req_head));
  uint8_t *ring = ring_req(base);
  uint64_t need = 0, pos = tail % cap;
  size_t taken = 0;
  for (const Frame &f : fr) {
    Layout L;
    layout_of(f.scheme, f.op, &L);
    if (L.req > cap) {
      if (taken == 0) return set_status(DPKEM_EINVAL);  // can never fit
      break;
    }
    if (cap - pos < L.req) {  // close the end with a PAD as soon as the PAD itself fits
      if (need + (cap - pos) > free) break;
      write_pad(ring + pos, cap - pos);
      need += cap - pos;
      pos = 0;
    }
    if (need + L.req > free) break;
    std::memcpy(ring + pos, frames + f.off, L.req);
    need += L.req;
    pos = (pos + L.req) % cap;
    taken = f.off + L.req;
  }
  if (need) st_rel(&c->req_tail, tail + need);
  *pushed = taken;
  return set_status(taken ? DPKEM_OK : DPKEM_EAGAIN);
}

int dpkem_ring_pop(void *base, uint8_t *out, size_t cap_out, size_t *got, size_t *n_frames) {
  dpkem_ring_control *c = ring_ctl(base);
  if (!c || !got || (!out && cap_out)) return set_status(DPKEM_EINVAL);
  *got = 0;
  if (n_frames) *n_frames = 0;
  const uint64_t cap = c->capacity, tail = ld_acq(&c->resp_tail);
  uint64_t head = c->resp_head;
  const uint8_t *ring = ring_resp(base, cap);
  size_t copied = 0, count = 0;
  while (head < tail) {
    dpkem_frame_header h;
    std::memcpy(&h, ring + head % cap, sizeof(h));
    if (h.frame_bytes < kHdr || h.frame_bytes % DPKEM_FRAME_ALIGN ||
        (h.magic != DPKEM_FRAME_PAD && h.magic != DPKEM_FRAME_MAGIC))
      return set_status(DPKEM_EINVAL);
    if (h.magic != DPKEM_FRAME_PAD) {
      if (copied + h.frame_bytes > cap_out) break;
      std::memcpy(out + copied, ring + head % cap, h.frame_bytes);
      copied += h.frame_bytes;
      count++;
    }
    head += h.frame_bytes;
  }
  st_rel(&c->resp_head, head);
  *got = copied;
  if (n_frames) *n_frames = count;
  return set_status(DPKEM_OK);
}

int dpkem_ring_acquire(void *base, size_t max_frames, size_t *req_off, size_t *req_bytes, size_t *req_advance,
                       size_t *resp_off, size_t *resp_bytes, size_t *resp_advance, size_t *n_frames) {
  dpkem_ring_control *c = ring_ctl(base);
  if (!c || !req_off || !req_bytes || !req_advance || !resp_off || !resp_bytes || !resp_advance || !n_frames)
    return set_status(DPKEM_EINVAL);
  Cursor cur{c->req_head, c->resp_tail, 0, 0};
  RingBatch b;
  const int rc = acquire_at(base, max_frames, &cur, &b);
  if (rc == DPKEM_EAGAIN && (cur.req_pending || cur.resp_pending)) publish(c, cur.req_pending, cur.resp_pending, 0);
  if (rc) return set_status(rc);
  *req_off = b.req_off;
  *req_bytes = b.req_bytes;
  *req_advance = b.req_advance;
  *resp_off = b.resp_off;
  *resp_bytes = b.resp_bytes;
  *resp_advance = b.resp_advance;
  *n_frames = b.n;
  return set_status(DPKEM_OK);
}

int dpkem_ring_release(void *base, size_t req_advance, size_t resp_advance, size_t n_frames) {
  dpkem_ring_control *c = ring_ctl(base);
  if (!c) return set_status(DPKEM_EINVAL);
  publish(c, req_advance, resp_advance, n_frames);
  return set_status(DPKEM_OK);
}

int dpkem_ring_serve(dpkem_ctx *const *ctxs, int nctx, int form, void *base, size_t max_frames, int idle_us) {
  dpkem_ring_control *c = ring_ctl(base);
  if (!ctxs || nctx < 1 || nctx > 16 || !c) return set_status(DPKEM_EINVAL);
  for (int k = 0; k < nctx; k++)
    if (!ctxs[k]) return set_status(DPKEM_EINVAL);
  const size_t cap = c->capacity;
  // Batches are acquired at the server's own cursors (ahead of the published counters),
  // run on the contexts in turn, and published strictly in acquisition order.
  Cursor cur{c->req_head, c->resp_tail, 0, 0};
  std::deque<std::pair<RingBatch, int>> inflight;
  int next = 0, rc = DPKEM_OK;
  while (true) {
    const bool stop = ld_acq(&c->stop) != 0;
    if (stop && inflight.empty()) break;
    if (!stop && (int)inflight.size() < nctx) {
      RingBatch b;
      rc = acquire_at(base, max_frames, &cur, &b);
      if (rc == DPKEM_OK) {
        size_t wrote = 0;
        rc = frames_submit(ctxs[next], form, ring_req(base) + b.req_off, b.req_bytes, ring_resp(base, cap) + b.resp_off,
                           b.resp_bytes, &wrote);
        if (rc) break;
        inflight.emplace_back(b, next);
        next = (next + 1) % nctx;
        continue;
      }
      if (rc != DPKEM_EAGAIN) break;
      rc = DPKEM_OK;
    }
    if (!inflight.empty()) {  // nothing new to start: retire the oldest batch
      const auto [b, k] = inflight.front();
      inflight.pop_front();
      if ((rc = frames_finish(ctxs[k])) != DPKEM_OK) break;
      publish(c, b.req_advance, b.resp_advance, b.n);
      continue;
    }
    if (cur.req_pending || cur.resp_pending) {  // PADs passed while idle
      publish(c, cur.req_pending, cur.resp_pending, 0);
      cur.req_pending = cur.resp_pending = 0;
    }
    if (idle_us > 0) usleep((useconds_t)idle_us);
  }
  for (auto &f : inflight) frames_finish(ctxs[f.second]);  // error path: let the copies land
  return set_status(rc);
}

}  // extern "C"
