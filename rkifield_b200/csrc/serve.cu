// serve.cu — the resident request loop (continuous batching).
//
// rkf_submit admits requests (camera renders, ray-cast batches, point-distance
// queries, CSG edits) against a device-memory budget and a slot limit;
// refused requests get RKF_BUSY.  A worker thread owns the device work: every
// time it wakes it takes the admitted requests (up to the next edit), gives
// each its device buffers from an arena, and launches them as one "tick" on
// the next of several streams: input copies, one persistent march launch for
// all renders and ray batches of the tick, point-query launches, output
// copies back to the caller's buffers, and an event.  Requests admitted while
// earlier ticks are still running go into a new tick on another stream right
// away, so their work overlaps on the device.
//
// Edits run in admission order: requests admitted before an edit are launched
// before it and read the old epoch of the brick index; requests admitted
// after it read the new one.  Edits are copy-on-write (edit.cu), so in-flight
// ticks are never disturbed.  The brick slots and index leaves an edit
// retires (the ones only older epochs reference) go back to their free lists
// two edits later: when the edit that creates epoch E + 2 starts, the slots
// and leaves retired at the creation of epoch E are reused, once every tick of
// an epoch before E has completed.  That point is fixed by the order of the
// edits alone, so slot numbers -- and so every output -- stay a function of
// the request and its epoch, and a session with an edit every few requests
// keeps its pool and leaf use bounded (brick_pool.rs:54,136 deallocate).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <unordered_map>

#include "../../include/rkf_cuda_testing.h"
#include "ctx.h"
#include "edit.h"
#include "march.h"

namespace rkf {

namespace {

size_t a256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// First-fit allocator over one device buffer (offsets in bytes).
struct Arena {
  DevBuf buf;
  std::map<size_t, size_t> free_;  // offset -> size
  rkf_status init(size_t bytes) {
    rkf_status st = buf.alloc(bytes);
    if (st != RKF_OK) return st;
    free_.clear();
    free_[0] = bytes;
    return RKF_OK;
  }
  bool alloc(size_t n, size_t* off) {
    n = a256(n);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        *off = it->first;
        const size_t rest = it->second - n;
        const size_t o = it->first + n;
        free_.erase(it);
        if (rest) free_[o] = rest;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t n) {
    n = a256(n);
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  char* at(size_t off) const { return buf.as<char>() + off; }
};

struct TicketRec {
  rkf_request req;
  rkf_result res;
  int state = 0;  // 0 pending, 1 launched, 2 done
  size_t bytes = 0;
};

struct Tick {
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<uint64_t> ids;
  std::vector<std::pair<size_t, size_t>> blocks;
  int pinned = -1;  // page-locked staging block of the segment table
  uint64_t epoch = 0;  // index epoch the tick's launches read
};

// Page-locked host blocks for segment tables: a copy from pageable memory
// may wait for the stream to drain before it is queued, which would hold the
// worker until an earlier tick on that stream finished.  A block returns to
// the pool when its tick completes.
struct PinnedPool {
  struct Block {
    void* p = nullptr;
    size_t cap = 0;
    bool used = false;
  };
  std::vector<Block> blocks;
  int get(size_t bytes) {
    for (size_t i = 0; i < blocks.size(); ++i)
      if (!blocks[i].used && blocks[i].cap >= bytes) {
        blocks[i].used = true;
        return static_cast<int>(i);
      }
    Block b;
    b.cap = std::max<size_t>(bytes, 64 << 10);
    if (cudaHostAlloc(&b.p, b.cap, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
    b.used = true;
    blocks.push_back(b);
    return static_cast<int>(blocks.size() - 1);
  }
  void put(int i) {
    if (i >= 0) blocks[static_cast<size_t>(i)].used = false;
  }
  // page-locked allocation waits for the device: make the usual blocks when
  // the session starts
  void reserve(int n, size_t bytes) {
    for (int i = 0; i < n; ++i) put(get(bytes));
  }
  void release() {  // every stream that read the blocks has been synchronised
    for (Block& b : blocks) cudaFreeHost(b.p);
    blocks.clear();
  }
};

double now_us(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
}

// Device bytes a request needs while in flight (inputs + outputs).
size_t request_bytes(const rkf_request& r) {
  switch (r.kind) {
    case RKF_REQ_RENDER:
      return a256(static_cast<size_t>(r.width) * r.height * 24) + 5 * 256;
    case RKF_REQ_RAYS:
      return a256(static_cast<size_t>(r.n) * 28) + a256(static_cast<size_t>(r.n) * 24) + 8 * 256;
    case RKF_REQ_POINTS:
      return a256(static_cast<size_t>(r.n) * 12) + a256(static_cast<size_t>(r.n) * 18) + 4 * 256;
    default:
      return 0;
  }
}

}  // namespace

struct ServeState {
  Ctx* c = nullptr;
  rkf_march_params p{};
  std::chrono::steady_clock::time_point t0;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::deque<uint64_t> pending;
  std::unordered_map<uint64_t, TicketRec> tickets;
  uint64_t next_id = 1;
  size_t budget = 0, reserved = 0;
  uint32_t inflight = 0;
  static constexpr int kStreams = 4;
  cudaStream_t streams[kStreams] = {};
  cudaStream_t edit_stream = nullptr;
  int next_stream = 0;
  Arena arena;
  PinnedPool pinned;
  std::deque<Tick> ticks;
  std::vector<DevBuf*> old_tops;
  // Top grid + field pairs for new epochs.  An edit writes its epoch into a
  // spare pair (a device allocation could wait for the ticks in flight); the
  // pair it replaces retires with the old epoch number and becomes a spare
  // once no tick of that epoch or earlier is in flight.
  std::vector<std::pair<DevBuf*, DevBuf*>> spares;
  std::vector<std::pair<uint64_t, std::pair<DevBuf*, DevBuf*>>> retiring;
  void recycle();
  // slots and leaves retired at the creation of `epoch`, not yet reusable
  struct Retired {
    uint64_t epoch;
    std::vector<uint32_t> slots, leaves;
  };
  std::deque<Retired> retired_q;
  void reclaim();
  rkf_status error = RKF_OK;
  std::string error_msg;

  void run();
  bool launch_tick(std::vector<uint64_t>& ids);
  void do_edit(uint64_t id);
  void poll_ticks();
};

// Returns to the free lists the slots and leaves retired at the creation of
// epochs up to c->epoch - 1, i.e. two or more edits before the one about to
// run (which would create c->epoch + 1), after waiting for the ticks of the
// epochs that read them.
void ServeState::reclaim() {
  while (!retired_q.empty() && retired_q.front().epoch + 1 <= c->epoch) {
    const Retired& r = retired_q.front();
    for (const Tick& t : ticks)
      if (t.epoch < r.epoch) cudaEventSynchronize(t.ev1);
    for (uint32_t slot : r.slots) c->free_slots.push_back(slot);
    for (uint32_t leaf : r.leaves) c->free_leaves.push_back(leaf);
    retired_q.pop_front();
  }
}

void ServeState::do_edit(uint64_t id) {
  rkf_edit_op op;
  {
    std::lock_guard<std::mutex> lk(mu);
    op = tickets[id].req.edit;
    tickets[id].res.start_us = now_us(t0);
    tickets[id].state = 1;
  }
  reclaim();
  EditOutcome out;
  std::pair<DevBuf*, DevBuf*> spare{nullptr, nullptr};
  if (!spares.empty()) {
    spare = spares.back();
    spares.pop_back();
    out.top_dst = spare.first->as<uint32_t>();
    out.field_dst = spare.second->as<uint8_t>();
  }
  // temporaries from the arena: freeing device memory would wait for every
  // tick in flight
  std::vector<std::pair<size_t, size_t>> taken;
  const EditScratch scratch = [&](size_t bytes) -> void* {
    size_t off;
    if (!arena.alloc(bytes, &off)) return nullptr;
    taken.emplace_back(off, bytes);
    return arena.at(off);
  };
  rkf_status st = apply_edit(c, op, edit_stream, &out, &scratch);
  cudaStreamSynchronize(edit_stream);  // error paths may return with work queued
  for (auto& t : taken) arena.release(t.first, t.second);
  if (st == RKF_OK && out.new_epoch && spare.first) {
    // the spare pair becomes the index; the old pair retires at this epoch
    std::swap(c->top.p, spare.first->p);
    std::swap(c->top.bytes, spare.first->bytes);
    std::swap(c->empty_dist.p, spare.second->p);
    std::swap(c->empty_dist.bytes, spare.second->bytes);
    retiring.push_back({c->epoch, spare});
    spare = {nullptr, nullptr};
    c->epoch++;
    retired_q.push_back({c->epoch, out.retired, out.retired_leaves});
  } else if (st == RKF_OK && out.new_epoch) {
    DevBuf* old = new DevBuf();
    std::swap(old->p, c->top.p);
    std::swap(old->bytes, c->top.bytes);
    std::swap(c->top.p, out.new_top.p);
    std::swap(c->top.bytes, out.new_top.bytes);
    old_tops.push_back(old);
    DevBuf* old_field = new DevBuf();
    std::swap(old_field->p, c->empty_dist.p);
    std::swap(old_field->bytes, c->empty_dist.bytes);
    std::swap(c->empty_dist.p, out.new_empty_dist.p);
    std::swap(c->empty_dist.bytes, out.new_empty_dist.bytes);
    old_tops.push_back(old_field);
    c->epoch++;
    retired_q.push_back({c->epoch, out.retired, out.retired_leaves});
  }
  if (spare.first) spares.push_back(spare);  // unused: no new epoch
  std::lock_guard<std::mutex> lk(mu);
  TicketRec& t = tickets[id];
  t.res.status = st;
  t.res.epoch = c->epoch;
  t.res.done_us = now_us(t0);
  t.state = 2;
  inflight--;
  cv_done.notify_all();
}

bool ServeState::launch_tick(std::vector<uint64_t>& ids) {
  if (ids.empty()) return true;
  cudaStream_t st = streams[next_stream];
  next_stream = (next_stream + 1) % kStreams;
  Tick tick;
  std::vector<Segment> segs;
  uint64_t first = 0;
  struct Pts { const float* in; float* d; float* g; uint16_t* m; uint32_t n; const rkf_request* r; };
  std::vector<Pts> pts;
  std::vector<std::pair<const rkf_request*, rkf_gbuffer>> renders;
  std::vector<std::pair<const rkf_request*, rkf_hits>> rays;
  const uint64_t epoch = c->epoch;
  tick.epoch = epoch;
  const double start = now_us(t0);
  for (uint64_t id : ids) {
    TicketRec* tr;
    {
      std::lock_guard<std::mutex> lk(mu);
      tr = &tickets[id];
      tr->state = 1;
      tr->res.start_us = start;
      tr->res.epoch = epoch;
    }
    const rkf_request& r = tr->req;
    size_t off;
    const size_t need = request_bytes(r);
    if (!arena.alloc(need, &off)) {
      std::lock_guard<std::mutex> lk(mu);
      tr->res.status = fail(RKF_OOM, "serve: request does not fit the device arena");
      tr->res.done_us = now_us(t0);
      tr->state = 2;
      reserved -= tr->bytes;
      inflight--;
      cv_done.notify_all();
      continue;
    }
    tick.blocks.emplace_back(off, need);
    tick.ids.push_back(id);
    char* b = arena.at(off);
    if (r.kind == RKF_REQ_RENDER) {
      const size_t n = static_cast<size_t>(r.width) * r.height;
      rkf_gbuffer g{};
      g.t = reinterpret_cast<float*>(b);
      b += a256(n * 4);
      g.normal = reinterpret_cast<float*>(b);
      b += a256(n * 12);
      g.slot = reinterpret_cast<uint32_t*>(b);
      b += a256(n * 4);
      g.material = reinterpret_cast<uint16_t*>(b);
      b += a256(n * 2);
      g.flags = reinterpret_cast<uint16_t*>(b);
      g.mem = RKF_MEM_DEVICE;
      Segment sg = view_segment(&r.camera, r.width, r.height, c->tuning.tile_w, c->tuning.tile_h, g);
      sg.first = first;
      first += sg.n_ids;
      segs.push_back(sg);
      renders.emplace_back(&r, g);
    } else if (r.kind == RKF_REQ_RAYS) {
      const size_t n = r.n;
      float* o = reinterpret_cast<float*>(b);
      b += a256(n * 12);
      float* d = reinterpret_cast<float*>(b);
      b += a256(n * 12);
      float* tm = reinterpret_cast<float*>(b);
      b += a256(n * 4);
      cudaMemcpyAsync(o, r.in0, n * 12, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d, r.in1, n * 12, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(tm, r.in2, n * 4, cudaMemcpyHostToDevice, st);
      rkf_hits h{};
      h.t = reinterpret_cast<float*>(b);
      b += a256(n * 4);
      h.flags = reinterpret_cast<uint16_t*>(b);
      b += a256(n * 2);
      if (r.mode == RKF_TRACE_CLOSEST) {
        h.normal = reinterpret_cast<float*>(b);
        b += a256(n * 12);
        h.slot = reinterpret_cast<uint32_t*>(b);
        b += a256(n * 4);
        h.material = reinterpret_cast<uint16_t*>(b);
      }
      h.mem = RKF_MEM_DEVICE;
      Segment sg = ray_segment(o, d, tm, static_cast<uint32_t>(n), r.mode, h);
      sg.first = first;
      first += sg.n_ids;
      segs.push_back(sg);
      rays.emplace_back(&r, h);
    } else {
      const size_t n = r.n;
      float* in = reinterpret_cast<float*>(b);
      b += a256(n * 12);
      cudaMemcpyAsync(in, r.in0, n * 12, cudaMemcpyHostToDevice, st);
      Pts q{in, reinterpret_cast<float*>(b), nullptr, nullptr, r.n, &r};
      b += a256(n * 4);
      q.g = reinterpret_cast<float*>(b);
      b += a256(n * 12);
      q.m = reinterpret_cast<uint16_t*>(b);
      pts.push_back(q);
    }
  }
  cudaEventCreate(&tick.ev0);
  cudaEventCreate(&tick.ev1);
  cudaEventRecord(tick.ev0, st);
  rkf_status lst = RKF_OK;
  if (!segs.empty()) {
    size_t off;
    const size_t need = sizeof(Segment) * segs.size() + 256;
    if (arena.alloc(need, &off)) {
      tick.blocks.emplace_back(off, need);
      Segment* dev_segs = reinterpret_cast<Segment*>(arena.at(off) + 256);
      const size_t sb = sizeof(Segment) * segs.size();
      tick.pinned = pinned.get(sb);
      bool uploaded = false;
      if (tick.pinned >= 0) {
        void* hp = pinned.blocks[static_cast<size_t>(tick.pinned)].p;
        std::memcpy(hp, segs.data(), sb);
        uploaded = cudaMemcpyAsync(dev_segs, hp, sb, cudaMemcpyHostToDevice, st) == cudaSuccess;
      }
      lst = launch_persistent_scratch(c, segs.data(), static_cast<uint32_t>(segs.size()), first, &p, c->tuning,
                                      st, dev_segs, reinterpret_cast<unsigned long long*>(arena.at(off)),
                                      uploaded, true);
    } else {
      lst = fail(RKF_OOM, "serve: no arena room for the segment table");
    }
  }
  for (const Pts& q : pts)
    if (lst == RKF_OK) lst = launch_query(c, q.in, q.n, q.d, q.g, q.m, st);
  for (auto& rg : renders) {
    const rkf_request& r = *rg.first;
    const size_t n = static_cast<size_t>(r.width) * r.height;
    if (r.out_t) cudaMemcpyAsync(r.out_t, rg.second.t, n * 4, cudaMemcpyDeviceToHost, st);
    if (r.out_normal) cudaMemcpyAsync(r.out_normal, rg.second.normal, n * 12, cudaMemcpyDeviceToHost, st);
    if (r.out_slot) cudaMemcpyAsync(r.out_slot, rg.second.slot, n * 4, cudaMemcpyDeviceToHost, st);
    if (r.out_material) cudaMemcpyAsync(r.out_material, rg.second.material, n * 2, cudaMemcpyDeviceToHost, st);
    if (r.out_flags) cudaMemcpyAsync(r.out_flags, rg.second.flags, n * 2, cudaMemcpyDeviceToHost, st);
  }
  for (auto& rh : rays) {
    const rkf_request& r = *rh.first;
    const size_t n = r.n;
    if (r.out_t) cudaMemcpyAsync(r.out_t, rh.second.t, n * 4, cudaMemcpyDeviceToHost, st);
    if (r.out_flags) cudaMemcpyAsync(r.out_flags, rh.second.flags, n * 2, cudaMemcpyDeviceToHost, st);
    if (r.mode == RKF_TRACE_CLOSEST) {
      if (r.out_normal) cudaMemcpyAsync(r.out_normal, rh.second.normal, n * 12, cudaMemcpyDeviceToHost, st);
      if (r.out_slot) cudaMemcpyAsync(r.out_slot, rh.second.slot, n * 4, cudaMemcpyDeviceToHost, st);
      if (r.out_material) cudaMemcpyAsync(r.out_material, rh.second.material, n * 2, cudaMemcpyDeviceToHost, st);
    }
  }
  for (const Pts& q : pts) {
    const rkf_request& r = *q.r;
    if (r.out_t) cudaMemcpyAsync(r.out_t, q.d, q.n * 4ull, cudaMemcpyDeviceToHost, st);
    if (r.out_normal) cudaMemcpyAsync(r.out_normal, q.g, q.n * 12ull, cudaMemcpyDeviceToHost, st);
    if (r.out_material) cudaMemcpyAsync(r.out_material, q.m, q.n * 2ull, cudaMemcpyDeviceToHost, st);
  }
  cudaEventRecord(tick.ev1, st);
  if (lst != RKF_OK) {
    std::lock_guard<std::mutex> lk(mu);
    error = lst;
    error_msg = rkf_last_error();
  }
  ticks.push_back(std::move(tick));
  return true;
}

void ServeState::poll_ticks() {
  while (!ticks.empty()) {
    // ticks on different streams may finish out of order: finalise any done
    bool progressed = false;
    for (auto it = ticks.begin(); it != ticks.end();) {
      if (cudaEventQuery(it->ev1) != cudaSuccess) {
        ++it;
        continue;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, it->ev0, it->ev1);
      const double done = now_us(t0);
      for (auto& bl : it->blocks) arena.release(bl.first, bl.second);
      pinned.put(it->pinned);
      {
        std::lock_guard<std::mutex> lk(mu);
        for (uint64_t id : it->ids) {
          auto tt = tickets.find(id);
          if (tt == tickets.end()) continue;
          tt->second.res.status = error;
          tt->second.res.done_us = done;
          tt->second.res.device_ms = ms;
          tt->second.state = 2;
          reserved -= tt->second.bytes;
          inflight--;
        }
      }
      cv_done.notify_all();
      cudaEventDestroy(it->ev0);
      cudaEventDestroy(it->ev1);
      it = ticks.erase(it);
      progressed = true;
    }
    if (!progressed) break;
  }
  recycle();
}

void ServeState::recycle() {
  uint64_t oldest = ~0ull;
  for (const Tick& t : ticks) oldest = std::min(oldest, t.epoch);
  for (auto it = retiring.begin(); it != retiring.end();) {
    if (it->first < oldest) {
      spares.push_back(it->second);
      it = retiring.erase(it);
    } else {
      ++it;
    }
  }
}

void ServeState::run() {
  cudaSetDevice(c->device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    if (stop && pending.empty() && ticks.empty()) break;
    // take everything admitted so far, up to (not including) the next edit
    std::vector<uint64_t> batch;
    uint64_t edit_id = 0;
    while (!pending.empty()) {
      const uint64_t id = pending.front();
      if (tickets[id].req.kind == RKF_REQ_EDIT) {
        if (batch.empty()) {
          edit_id = id;
          pending.pop_front();
        }
        break;
      }
      batch.push_back(id);
      pending.pop_front();
    }
    lk.unlock();
    if (edit_id) do_edit(edit_id);
    if (!batch.empty()) launch_tick(batch);
    poll_ticks();
    lk.lock();
    if (pending.empty() && !stop) {
      if (ticks.empty())
        cv_work.wait(lk, [&] { return stop || !pending.empty(); });
      else
        cv_work.wait_for(lk, std::chrono::microseconds(20));
    }
  }
}

}  // namespace rkf

using namespace rkf;

extern "C" {

rkf_status rkf_serve_start(rkf_ctx* ctx, const rkf_march_params* p) {
  if (!ctx || !p) return fail(RKF_INVALID_ARG, "rkf_serve_start: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (c->serve) return fail(RKF_BUSY, "rkf_serve_start: already serving");
  if (c->obj_count() == 0) return fail(RKF_INVALID_ARG, "rkf_serve_start: the scene has no objects");
  if (p->strategy != RKF_STRATEGY_BRUTE)
    return fail(RKF_UNSUPPORTED, "rkf_serve_start: serving marches with the brute strategy only");
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  RKF_CUDA_TRY(cudaStreamSynchronize(c->stream));
  auto* s = new ServeState();
  s->c = c;
  s->p = *p;
  s->t0 = std::chrono::steady_clock::now();
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  s->budget = c->cfg.mem_budget_bytes ? c->cfg.mem_budget_bytes : std::min<size_t>(free_b / 4, 8ull << 30);
  rkf_status st = s->arena.init(s->budget + (64ull << 20));
  // reserve index room for the session's edits so the leaves never move
  if (st == RKF_OK) st = c->ensure_leaf_capacity(c->n_leaves + 65536);
  if (st != RKF_OK) {
    delete s;
    return st;
  }
  for (auto& strm : s->streams) cudaStreamCreateWithFlags(&strm, cudaStreamNonBlocking);
  // edits hold up every request behind them: their small kernels take free
  // SM slots ahead of queued ticks
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  cudaStreamCreateWithPriority(&s->edit_stream, cudaStreamNonBlocking, prio_high);
  s->pinned.reserve(2 * ServeState::kStreams, 256 << 10);
  for (int i = 0; i < 2; ++i) {
    auto* tp = new DevBuf();
    auto* fp = new DevBuf();
    if (tp->alloc(std::max<uint64_t>(c->top_len, 1) * 4) == RKF_OK &&
        fp->alloc(std::max<uint64_t>(c->top_len, 1)) == RKF_OK) {
      s->spares.push_back({tp, fp});
    } else {  // no spares: edits allocate their epochs
      delete tp;
      delete fp;
      cudaGetLastError();
    }
  }
  c->leaves_frozen = true;
  c->serve = s;
  s->worker = std::thread([s] { s->run(); });
  return RKF_OK;
}

rkf_status rkf_serve_stop(rkf_ctx* ctx) {
  if (!ctx) return fail(RKF_INVALID_ARG, "rkf_serve_stop: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  ServeState* s = c->serve;
  if (!s) return RKF_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->worker.join();
  for (auto& strm : s->streams) {
    cudaStreamSynchronize(strm);
    cudaStreamDestroy(strm);
  }
  cudaStreamSynchronize(s->edit_stream);
  cudaStreamDestroy(s->edit_stream);
  s->pinned.release();
  for (DevBuf* d : s->old_tops) delete d;
  for (auto& pr : s->spares) {
    delete pr.first;
    delete pr.second;
  }
  for (auto& r : s->retiring) {
    delete r.second.first;
    delete r.second.second;
  }
  // every stream is idle: what is still held is free now (apply_edit already
  // took retired slots out of used_slots)
  for (const ServeState::Retired& r : s->retired_q) {
    for (uint32_t slot : r.slots) c->free_slots.push_back(slot);
    for (uint32_t leaf : r.leaves) c->free_leaves.push_back(leaf);
  }
  c->leaves_frozen = false;
  c->serve = nullptr;
  delete s;
  return RKF_OK;
}

rkf_status rkf_submit(rkf_ctx* ctx, const rkf_request* req, rkf_ticket* ticket) {
  if (!ctx || !req || !ticket) return fail(RKF_INVALID_ARG, "rkf_submit: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  ServeState* s = c->serve;
  if (!s) return fail(RKF_INVALID_ARG, "rkf_submit: the context is not serving (rkf_serve_start)");
  switch (req->kind) {
    case RKF_REQ_RENDER:
      if (req->width == 0 || req->height == 0) return fail(RKF_INVALID_ARG, "rkf_submit: empty render");
      break;
    case RKF_REQ_RAYS:
      if (req->n == 0 || !req->in0 || !req->in1 || !req->in2 || req->mode > RKF_TRACE_SHADOW || !req->out_t)
        return fail(RKF_INVALID_ARG, "rkf_submit: bad ray request");
      break;
    case RKF_REQ_POINTS:
      if (req->n == 0 || !req->in0) return fail(RKF_INVALID_ARG, "rkf_submit: bad point request");
      break;
    case RKF_REQ_EDIT:
      break;
    default:
      return fail(RKF_INVALID_ARG, "rkf_submit: unknown request kind");
  }
  const size_t need = request_bytes(*req);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return fail(RKF_BUSY, "rkf_submit: the loop is stopping");
  if (s->inflight >= c->cfg.max_inflight || s->reserved + need > s->budget)
    return fail(RKF_BUSY, "rkf_submit: no free slot or memory budget");
  const uint64_t id = s->next_id++;
  TicketRec& t = s->tickets[id];
  t.req = *req;
  t.bytes = need;
  std::memset(&t.res, 0, sizeof(t.res));
  t.res.kind = req->kind;
  t.res.submit_us = now_us(s->t0);
  s->reserved += need;
  s->inflight++;
  s->pending.push_back(id);
  *ticket = id;
  s->cv_work.notify_one();
  return RKF_OK;
}

rkf_status rkf_poll(rkf_ctx* ctx, rkf_ticket ticket, rkf_result* out, uint32_t timeout_us) {
  if (!ctx || !out) return fail(RKF_INVALID_ARG, "rkf_poll: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  ServeState* s = c->serve;
  if (!s) return fail(RKF_INVALID_ARG, "rkf_poll: the context is not serving");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return fail(RKF_INVALID_ARG, "rkf_poll: unknown ticket");
  if (it->second.state != 2 && timeout_us) {
    s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), [&] {
      auto jt = s->tickets.find(ticket);
      return jt == s->tickets.end() || jt->second.state == 2;
    });
    it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return fail(RKF_INVALID_ARG, "rkf_poll: unknown ticket");
  }
  if (it->second.state != 2)
    return timeout_us ? fail(RKF_TIMEOUT, "rkf_poll: not complete") : RKF_NOT_READY;
  *out = it->second.res;
  s->tickets.erase(it);
  return RKF_OK;
}

rkf_status rkf_cancel(rkf_ctx* ctx, rkf_ticket ticket) {
  if (!ctx) return fail(RKF_INVALID_ARG, "rkf_cancel: null argument");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  ServeState* s = c->serve;
  if (!s) return fail(RKF_INVALID_ARG, "rkf_cancel: the context is not serving");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return fail(RKF_INVALID_ARG, "rkf_cancel: unknown ticket");
  if (it->second.state != 0) return fail(RKF_BUSY, "rkf_cancel: the request is already running");
  for (auto p = s->pending.begin(); p != s->pending.end(); ++p)
    if (*p == ticket) {
      s->pending.erase(p);
      break;
    }
  it->second.state = 2;
  it->second.res.status = RKF_CANCELLED;
  it->second.res.done_us = now_us(s->t0);
  s->reserved -= it->second.bytes;
  s->inflight--;
  s->cv_done.notify_all();
  return RKF_OK;
}

}  // extern "C"

extern "C" rkf_status rkf_testing_pool_state(rkf_ctx* ctx, uint32_t out[5]) {
  if (!ctx || !out) return fail(RKF_INVALID_ARG, "rkf_testing_pool_state: null argument");
  const Ctx* c = reinterpret_cast<const Ctx*>(ctx);
  out[0] = c->capacity;
  out[1] = c->used_slots;
  out[2] = static_cast<uint32_t>(c->free_slots.size());
  out[3] = c->n_leaves;
  out[4] = static_cast<uint32_t>(c->free_leaves.size());
  return RKF_OK;
}
