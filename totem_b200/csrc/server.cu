// Serving runtime: a resident scheduler with continuous batching (totem_server_* in
// include/totem_b200.h).  No counterpart in the reference, whose entry point serves one blocking
// request at a time (waveCuda.cpp:4-101) and allocates and frees all device state per call
// (cuda_source_lobato.cu:1018-1562).
//
// Three host threads per server:
//   prep      admission against the memory budget, then upload and transmission build of one
//             request at a time on the request's own stream (overlapping the running slice loop);
//   schedule  the tick loop: every tick starts the probe groups the Planner admits, advances all
//             running groups by one slice (one k_row_groups and one k_col_groups launch per window
//             size, on the server stream), reduces the detector sums of finished groups and
//             combines the results of finished requests;
//   complete  copies results into the caller's buffers and retires the request's device state.
// Device memory comes from a dedicated stream-ordered pool, so admitting and retiring requests
// never synchronises the device.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "planner.h"
#include "session.h"

using totem::Status;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

bool fused_window(int h, int w) { return h == w && totem::fused_window_ok(h); }

struct Request {
  unsigned long long ticket = 0;
  TotemStemArgs args{};
  TotemStemOut out{};
  int state = TOTEM_REQ_QUEUED;
  int status = TOTEM_OK;
  std::string error;
  Clock::time_point t_submit, t_admit, t_ready, t_done;
  size_t reserve = 0;               // resident footprint held against the budget
  totem_session* sess = nullptr;
  cudaEvent_t ready = nullptr;      // transmission built (session stream)
  cudaEvent_t handoff = nullptr;    // detector sums complete (server stream)
  cudaEvent_t done = nullptr;       // results combined (session stream)
  totem::DetectionEvents de;
  long long items = 0, items_left = 0;
  int nblk = 0;
  int skip_band = 0;                // its groups leave out the propagator's zero band
  size_t item_bytes = 0;
  long long probe_slices = 0;
  double est = 0;                   // estimated device seconds (preparation order)
  int lane = 1;                     // 0 fast, 1 bulk
};

// A tick loop: its own planner, tick counter, stream and staging ring.  Lane 0 (fast) takes the
// requests whose probe waves fit it whole and runs on the highest stream priority, so a small
// request advances one slice per short tick instead of one slice per tick of the large requests
// beside it; lane 1 (bulk) takes the rest.  Both lanes' launches run concurrently on the device.
struct Lane {
  totem::Planner planner;
  cudaStream_t st = nullptr;
  int tick = 0;
  char* h_stage = nullptr;          // pinned [K][slot_bytes]
  char* d_stage = nullptr;          // device [K][slot_bytes]
  std::vector<cudaEvent_t> tick_ev;
  size_t wave = 0;
  Lane(size_t wave_bytes, size_t chunk, int policy, size_t max_groups)
      : planner(wave_bytes, chunk, policy, max_groups), wave(wave_bytes) {}
};

// Resident bytes of a request outside its probe waves (upper estimate, pool slack included).
size_t resident_bytes(const TotemStemArgs& a) {
  const size_t plane = (size_t)a.p_height * a.p_width;
  const size_t vol = (size_t)a.height * a.width;
  size_t b = plane * (size_t)std::max(a.slices, 1) * 8;  // transmission stack
  b += plane * (8 + 4 + 4);                             // s2, aper_true, general kx/ky share
  b += plane * (size_t)std::max(a.cim_len, 0) * 4;
  long long atoms = 0;
  for (const double* cnt : {a.atom_slice, a.atom_slice_i, a.series_n_corr, a.series_n_i_corr})
    if (cnt)
      for (int s = 0; s < a.slices; ++s) atoms += (long long)cnt[s];
  b += (size_t)atoms * (16 + 26 * 4 + 40);
  b += vol * 8 * ((size_t)a.w_num + 1);                  // probes, propagator
  b += vol * 4 * 2 * (size_t)std::max(a.aper_num, 1);    // masks
  const size_t ad = (size_t)std::max(a.aper_num, 0) * std::max(a.depth, 0);
  const size_t events = (size_t)std::max(a.layer_len, 0) + 1;
  b += ad * 8 * (events * (size_t)a.w_num + events);     // acc + outputs
  return b + (32u << 20);
}

// Estimated device time of a request in seconds, for ordering preparation under the SHORTEST
// policy: slice loop ~7.2 ps per probe-slice pixel, transmission build ~1.6 ps per atom-pixel
// (SrTiO3 on B200: 1.9 us per probe-slice at 512^2; 27 ms for 16 000 atoms on a 1024^2 grid).
double est_seconds(const TotemStemArgs& a) {
  long long atoms = 0;
  for (const double* cnt : {a.atom_slice, a.atom_slice_i})
    if (cnt)
      for (int s = 0; s < a.slices; ++s) atoms += (long long)cnt[s];
  const double loop = 7.2e-12 * (double)a.w_num * a.depth * a.slices * (double)a.height * a.width;
  const double tx = 1.6e-12 * (double)atoms * a.p_height * a.p_width;
  return loop + tx;
}

}  // namespace

struct totem_server {
  int device = 0;
  TotemServerOptions opt{};
  cudaMemPool_t pool = nullptr;
  std::vector<std::unique_ptr<Lane>> lanes;
  size_t static_budget = 0, static_used = 0;

  std::mutex mu;
  std::condition_variable cv;       // any state change
  std::deque<Request*> submitted, ready, completing;
  std::map<unsigned long long, std::unique_ptr<Request>> reqs;
  std::map<unsigned long long, Request*> running;
  unsigned long long next_ticket = 1;
  bool stopping = false, prep_exited = false, sched_exited = false;
  int prep_live = 0;                // prep threads still running
  Status fatal;

  std::vector<std::thread> prep_thrs;
  std::thread sched_thr, done_thr;

  // scheduler-owned device state
  std::map<int, std::unique_ptr<totem::DevBuf>> tw;  // stage twiddles per window size
  int K = 4;                                         // ticks queued ahead
  size_t slot_bytes = 0;
  size_t max_groups = 4096;
  TotemServerStats stats{};  // guarded by mu

  Status init();
  void prep_loop();
  void sched_loop();
  void done_loop();
  Status prepare(Request* r);
  Status tick_once(Lane& lane, bool* progressed);
  Status lookup(unsigned long long ticket, Request** r);
  Status complete_request(Request* r);
  void fail_request(Request* r, const Status& s);
  void fail_all(const Status& s);
};

Status totem_server::init() {
  TOTEM_CUDA(cudaSetDevice(device));
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  TOTEM_CUDA(cudaMemPoolCreate(&pool, &props));
  unsigned long long keep = ~0ull;  // keep freed memory in the pool for the next request
  TOTEM_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  size_t fr = 0, tot = 0;
  TOTEM_CUDA(cudaMemGetInfo(&fr, &tot));
  size_t budget = opt.hbm_budget ? (size_t)opt.hbm_budget : (size_t)(0.9 * (double)fr);
  size_t wave = opt.wave_bytes ? (size_t)opt.wave_bytes : std::min<size_t>(1ull << 30, budget / 4);
  if (wave >= budget) return Status::Err(TOTEM_ERR_INVALID_ARG, "wave_bytes must be below hbm_budget");
  opt.hbm_budget = budget;
  opt.wave_bytes = wave;
  if (!opt.chunk_bytes) opt.chunk_bytes = wave / 4;
  static_budget = budget - wave;
  K = opt.ticks_ahead > 0 ? opt.ticks_ahead : 4;
  // per window size: descriptors, launch-item prefix, alignment; the mixed launch adds a second
  // prefix and two queue counters
  slot_bytes = max_groups * (sizeof(totem::GroupDesc) + 2 * sizeof(int)) + 64 * (sizeof(int) + 256) + 1024;
  // Tick streams run above the default priority of the preparation streams, so slice steps of
  // running requests are not queued behind transmission builds; the fast lane above the bulk lane.
  int least = 0, greatest = 0;
  TOTEM_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  const size_t fast_wave = std::min<size_t>(256ull << 20, wave / 4);
  for (int l = 0; l < 2; ++l) {
    const size_t w = l == 0 ? fast_wave : wave;
    lanes.emplace_back(new Lane(w, l == 0 ? w : opt.chunk_bytes, opt.policy, max_groups));
    Lane& ln = *lanes.back();
    const int prio = l == 0 ? greatest : std::min(least, greatest + 1);
    TOTEM_CUDA(cudaStreamCreateWithPriority(&ln.st, cudaStreamNonBlocking, prio));
    TOTEM_CUDA(cudaMallocHost(&ln.h_stage, slot_bytes * K));
    TOTEM_CUDA(cudaMalloc(&ln.d_stage, slot_bytes * K));
    ln.tick_ev.assign(K, nullptr);
    // blocking-sync events: a thread waiting for the device sleeps instead of spinning on a core
    // that the preparation thread needs
    for (auto& e : ln.tick_ev)
      TOTEM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming | cudaEventBlockingSync));
  }
  // Map the pool's memory once up front (the waves plus a few transmission stacks): growing a
  // pool maps new physical memory, which took tens of milliseconds per request when request
  // sizes grew; freed memory stays in the pool (release threshold) for suballocation.
  const size_t reserve = std::min<size_t>(budget, wave + (4ull << 30));
  void* warm = nullptr;
  TOTEM_CUDA(cudaMallocFromPoolAsync(&warm, reserve, pool, lanes[1]->st));
  TOTEM_CUDA(cudaFreeAsync(warm, lanes[1]->st));
  TOTEM_CUDA(cudaStreamSynchronize(lanes[1]->st));
  return Status::Ok();
}

void totem_server::fail_request(Request* r, const Status& s) {
  // caller holds ``mu``
  r->state = TOTEM_REQ_FAILED;
  r->status = s.code;
  r->error = s.msg;
  r->t_done = Clock::now();
}

void totem_server::fail_all(const Status& s) {
  std::lock_guard<std::mutex> lk(mu);
  if (fatal.ok()) fatal = s;
  for (auto& kv : reqs)
    if (kv.second->state != TOTEM_REQ_DONE && kv.second->state != TOTEM_REQ_FAILED) fail_request(kv.second.get(), s);
  submitted.clear();
  ready.clear();
  running.clear();
  cv.notify_all();
}

// ---------------------------------------------------------------------------------------------
// prep: admission, upload, transmission build
// ---------------------------------------------------------------------------------------------
Status totem_server::prepare(Request* r) {
  if (totem::inject_prepare_failure())
    return Status::Err(TOTEM_ERR_STATE, "injected failure of the request's preparation");
  TOTEM_CUDA(cudaSetDevice(device));
  totem_session* s = nullptr;
  TOTEM_TRY(totem::create_session(device, nullptr, &s));
  r->sess = s;
  s->use_pool(pool);
  TOTEM_TRY(s->upload_args(&r->args, true));
  int launches = 0;
  TOTEM_TRY(s->build_transmission(TOTEM_PATH_FUSED, &launches));
  r->de = s->detection_events();
  TOTEM_TRY(totem::upload(s->ev_slice, r->de.event_of_slice, s->stream));
  const size_t ad = (size_t)s->aper_num * s->depth;
  const size_t L = s->mid_layer.size();
  const size_t acc_n = (size_t)r->de.n_events * s->w_num * ad;
  TOTEM_TRY(s->acc.ensure(std::max<size_t>(acc_n, 1) * sizeof(double)));
  if (acc_n) TOTEM_CUDA(cudaMemsetAsync(s->acc.p, 0, acc_n * sizeof(double), s->stream));
  TOTEM_TRY(s->out_result.ensure(std::max<size_t>(ad, 1) * sizeof(double)));
  TOTEM_TRY(s->out_mid.ensure(std::max<size_t>(ad * L, 1) * sizeof(double)));
  r->items = (s->aper_num > 0) ? (long long)s->w_num * s->depth : 0;
  r->items_left = r->items;
  r->nblk = totem::col_blocks(s->h);
  r->skip_band = (totem::band_skip_enabled() && totem::band_skip_ok(s->h, s->band, 0)) ? 1 : 0;
  r->item_bytes = (size_t)s->h * s->w * sizeof(float2) + (size_t)r->de.n_events * s->aper_num * r->nblk * sizeof(double);
  r->probe_slices = (long long)s->w_num * s->depth * s->slices;
  TOTEM_CUDA(cudaEventCreateWithFlags(&r->ready, cudaEventDisableTiming));
  TOTEM_CUDA(cudaEventCreateWithFlags(&r->handoff, cudaEventDisableTiming));
  TOTEM_CUDA(cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming | cudaEventBlockingSync));
  TOTEM_CUDA(cudaEventRecord(r->ready, s->stream));
  return Status::Ok();
}

void totem_server::prep_loop() {
  cudaSetDevice(device);
  for (;;) {
    Request* r = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv.wait(lk, [&] { return !submitted.empty() || stopping || !fatal.ok(); });
      if (submitted.empty() || !fatal.ok()) break;
      // FIFO prepares in arrival order; SHORTEST prepares the cheapest queued request first
      auto pick = submitted.begin();
      if (opt.policy == TOTEM_SCHED_SHORTEST)
        pick = std::min_element(submitted.begin(), submitted.end(),
                                [](const Request* a, const Request* b) { return a->est < b->est; });
      r = *pick;
      submitted.erase(pick);
      // a request larger than the whole budget is admitted alone
      cv.wait(lk, [&] {
        return static_used + r->reserve <= static_budget || static_used == 0 || !fatal.ok();
      });
      if (!fatal.ok()) break;
      static_used += r->reserve;
      r->state = TOTEM_REQ_PREPARING;
      r->t_admit = Clock::now();
    }
    const Status st = prepare(r);
    std::lock_guard<std::mutex> lk(mu);
    if (!st.ok()) {
      fail_request(r, st);
      if (r->sess) {
        cudaStreamSynchronize(r->sess->stream);
        delete r->sess;
        r->sess = nullptr;
      }
      static_used -= r->reserve;
    } else {
      ready.push_back(r);
    }
    cv.notify_all();
  }
  std::lock_guard<std::mutex> lk(mu);
  if (--prep_live == 0) prep_exited = true;
  cv.notify_all();
}

// ---------------------------------------------------------------------------------------------
// schedule: the tick loop
// ---------------------------------------------------------------------------------------------
Status totem_server::complete_request(Request* r) {
  totem_session* s = r->sess;
  TOTEM_CUDA(cudaEventRecord(r->handoff, lanes[r->lane]->st));
  TOTEM_CUDA(cudaStreamWaitEvent(s->stream, r->handoff, 0));
  int launches = 0;
  if (r->items > 0) TOTEM_TRY(s->combine_results(r->de, &launches));
  s->has_result = true;
  s->last_what = 0;
  TOTEM_CUDA(cudaEventRecord(r->done, s->stream));
  std::lock_guard<std::mutex> lk(mu);
  running.erase(r->ticket);
  completing.push_back(r);
  cv.notify_all();
  return Status::Ok();
}

// The running request of a probe group (every group's request stays in ``running`` until its last
// group finished; a miss is an internal error, reported rather than thrown).
Status totem_server::lookup(unsigned long long ticket, Request** r) {
  std::lock_guard<std::mutex> lk(mu);
  auto it = running.find(ticket);
  if (it == running.end()) return Status::Err(TOTEM_ERR_STATE, "scheduler: probe group of an unknown request");
  *r = it->second;
  return Status::Ok();
}

Status totem_server::tick_once(Lane& lane, bool* progressed) {
  *progressed = false;
  totem::Planner& planner = lane.planner;
  const int tick = lane.tick;
  cudaStream_t sst = lane.st;
  const int slot = tick % K;
  const Clock::time_point t0 = Clock::now();
  TOTEM_CUDA(cudaEventSynchronize(lane.tick_ev[slot]));  // tick - K has finished: its slot is free
  const Clock::time_point t1 = Clock::now();
  long long launched = 0, advanced = 0;
  // start the admitted groups
  std::vector<totem::PlanGroup> started = planner.start(tick);
  for (const totem::PlanGroup& g : started) {
    Request* r = nullptr;
    TOTEM_TRY(lookup(g.req, &r));
    void* psi = nullptr;
    void* part = nullptr;
    TOTEM_CUDA(cudaMallocFromPoolAsync(&psi, (size_t)g.items * g.n * g.n * sizeof(float2), pool, sst));
    const size_t pb = (size_t)r->de.n_events * g.items * r->sess->aper_num * r->nblk * sizeof(double);
    TOTEM_CUDA(cudaMallocFromPoolAsync(&part, std::max<size_t>(pb, 8), pool, sst));
    planner.attach(g, psi, part);
  }
  const std::vector<totem::PlanGroup>& act = planner.active();
  if (act.empty()) return Status::Ok();
  *progressed = true;
  for (const totem::PlanGroup& g : act) advanced += g.items;
  // one row and one column launch per window size over every active group
  std::map<int, std::vector<const totem::PlanGroup*>> by_n;
  for (const totem::PlanGroup& g : act) by_n[g.n].push_back(&g);
  char* h = lane.h_stage + (size_t)slot * slot_bytes;
  char* d = lane.d_stage + (size_t)slot * slot_bytes;
  size_t off = 0;
  auto twiddles_of = [&](int n, const float2** out) -> Status {
    auto& twb = tw[n];
    if (!twb) {
      twb.reset(new totem::DevBuf());
      TOTEM_TRY(totem::upload(*twb, totem::twiddles(n), sst));
      TOTEM_CUDA(cudaStreamSynchronize(sst));  // once per window size: the other lane may use it next
    }
    *out = twb->as<float2>();
    return Status::Ok();
  };
  auto describe = [&](const totem::PlanGroup& g, int n, totem::GroupDesc& x) -> Status {
    Request* r = nullptr;
    TOTEM_TRY(lookup(g.req, &r));
    const totem_session* s = r->sess;
    x.psi = static_cast<float2*>(g.psi);
    x.t_stack = s->T.as<float2>();
    x.probe = s->probe.as<float2>();
    x.prop = s->prop.as<float2>();
    x.mask_mid = s->mask_mid.as<float>();
    x.mask_exit = s->mask_exit.as<float>();
    x.part = static_cast<double*>(g.part);
    x.event_of_slice = s->ev_slice.as<int>();
    x.geo = totem::ScanGeom{s->begin_row, s->begin_col, s->step, s->width_red, s->depth, s->p_w};
    x.p_h = s->p_h;
    x.item0 = (int)g.item0;
    x.items = g.items;
    x.start_tick = g.start_tick;
    x.slices = s->slices;
    x.aper_num = s->aper_num;
    x.exit_event = r->de.exit_event;
    x.n = n;
    x.skip_band = r->skip_band;
    x.skip = r->skip_band ? totem::band_tiles(n, totem::col_blocks(n)) : totem::TileSkip();
    return Status::Ok();
  };
  // Several of the window sizes 256^2 .. 1024^2 at this tick: one persistent launch per pass for
  // all of them (TotemServerOptions.mixed_windows)
  int mixed_sizes = 0;
  for (auto& kv : by_n) mixed_sizes += totem::mixed_window_ok(kv.first) ? 1 : 0;
  if (opt.mixed_windows == 1 && mixed_sizes >= 2) {
    std::vector<const totem::PlanGroup*> gs;
    totem::MixedTwiddles mt{nullptr, nullptr, nullptr};
    for (auto it = by_n.begin(); it != by_n.end();) {
      if (!totem::mixed_window_ok(it->first)) {
        ++it;
        continue;
      }
      const float2* t = nullptr;
      TOTEM_TRY(twiddles_of(it->first, &t));
      (it->first == 256 ? mt.n256 : it->first == 512 ? mt.n512 : mt.n1024) = t;
      gs.insert(gs.end(), it->second.begin(), it->second.end());
      it = by_n.erase(it);
    }
    const size_t ng = gs.size();
    const size_t desc_off = off, rb_off = off + ng * sizeof(totem::GroupDesc), cb_off = rb_off + (ng + 1) * sizeof(int);
    const size_t q_off = cb_off + (ng + 1) * sizeof(int);
    off = q_off + 2 * sizeof(int);
    off = (off + 255) & ~(size_t)255;
    if (off > slot_bytes) return Status::Err(TOTEM_ERR_STATE, "scheduler staging slot overflow");
    auto* desc = reinterpret_cast<totem::GroupDesc*>(h + desc_off);
    auto* rb = reinterpret_cast<int*>(h + rb_off);
    auto* cbg = reinterpret_cast<int*>(h + cb_off);
    auto* q = reinterpret_cast<int*>(h + q_off);
    long long row_units = 0, col_units = 0;
    for (size_t i = 0; i < ng; ++i) {
      TOTEM_TRY(describe(*gs[i], gs[i]->n, desc[i]));
      rb[i] = (int)row_units;
      cbg[i] = (int)col_units;
      row_units += (long long)gs[i]->items * totem::mixed_units(gs[i]->n, true, desc[i].skip);
      col_units += (long long)gs[i]->items * totem::mixed_units(gs[i]->n, false, desc[i].skip);
    }
    if (row_units > INT32_MAX || col_units > INT32_MAX)
      return Status::Err(TOTEM_ERR_STATE, "too many work units in one mixed launch");
    rb[ng] = (int)row_units;
    cbg[ng] = (int)col_units;
    q[0] = q[1] = 0;
    TOTEM_CUDA(cudaMemcpyAsync(d + desc_off, h + desc_off, off - desc_off, cudaMemcpyHostToDevice, sst));
    const auto* dd = reinterpret_cast<const totem::GroupDesc*>(d + desc_off);
    int* dq = reinterpret_cast<int*>(d + q_off);
    TOTEM_TRY(totem::launch_mixed_groups(true, dd, reinterpret_cast<const int*>(d + rb_off), (int)ng, row_units, tick,
                                         mt, dq, sst));
    TOTEM_TRY(totem::launch_mixed_groups(false, dd, reinterpret_cast<const int*>(d + cb_off), (int)ng, col_units,
                                         tick, mt, dq + 1, sst));
    launched += 2;
  }
  for (auto& kv : by_n) {
    const int n = kv.first;
    const std::vector<const totem::PlanGroup*>& gs = kv.second;
    const float2* twn = nullptr;
    TOTEM_TRY(twiddles_of(n, &twn));
    const size_t ng = gs.size();
    const size_t desc_off = off, ib_off = off + ng * sizeof(totem::GroupDesc);
    off = ib_off + (ng + 1) * sizeof(int);
    off = (off + 255) & ~(size_t)255;
    if (off > slot_bytes) return Status::Err(TOTEM_ERR_STATE, "scheduler staging slot overflow");
    auto* desc = reinterpret_cast<totem::GroupDesc*>(h + desc_off);
    auto* ib = reinterpret_cast<int*>(h + ib_off);
    long long items = 0;
    // column tiles left out of the column launch: those in the zero band of every group
    const int nblk_n = totem::col_blocks(n);
    int skip_lo = 0, skip_hi = nblk_n;
    for (size_t i = 0; i < ng; ++i) {
      const totem::PlanGroup& g = *gs[i];
      totem::GroupDesc& x = desc[i];
      TOTEM_TRY(describe(g, n, x));
      skip_lo = std::max(skip_lo, x.skip.z0);
      skip_hi = std::min(skip_hi, x.skip.z0 + x.skip.nskip);
      ib[i] = (int)items;
      items += g.items;
    }
    ib[ng] = (int)items;
    TOTEM_CUDA(cudaMemcpyAsync(d + desc_off, h + desc_off, off - desc_off, cudaMemcpyHostToDevice, sst));
    const auto* dd = reinterpret_cast<const totem::GroupDesc*>(d + desc_off);
    const auto* dib = reinterpret_cast<const int*>(d + ib_off);
    TOTEM_TRY(totem::launch_row_groups(n, dd, dib, (int)ng, items, tick, twn, sst));
    totem::TileSkip skip;
    if (skip_hi > skip_lo) {
      skip.z0 = skip_lo;
      skip.nskip = skip_hi - skip_lo;
    }
    TOTEM_TRY(totem::launch_col_groups(n, dd, dib, (int)ng, items, tick, twn, skip, sst));
    launched += 2;
  }
  // groups that ran their last slice: detector sums, then their wave memory goes back
  for (const totem::PlanGroup& g : planner.finish(tick)) {
    Request* r = nullptr;
    TOTEM_TRY(lookup(g.req, &r));
    const totem_session* s = r->sess;
    const long ad = (long)s->aper_num * s->depth;
    const size_t estride = (size_t)g.items * s->aper_num * r->nblk;
    for (int e = 0; e < r->de.n_events; ++e)
      TOTEM_TRY(totem::launch_det_reduce(static_cast<const double*>(g.part) + e * estride, r->nblk, s->aper_num,
                                         g.items, (int)g.item0, s->depth,
                                         s->acc.as<double>() + (size_t)e * s->w_num * ad, sst,
                                         r->skip_band ? totem::band_tiles(s->h, r->nblk) : totem::TileSkip()));
    launched += r->de.n_events;
    TOTEM_CUDA(cudaFreeAsync(g.psi, sst));
    TOTEM_CUDA(cudaFreeAsync(g.part, sst));
    r->items_left -= g.items;
    if (r->items_left == 0) TOTEM_TRY(complete_request(r));
  }
  TOTEM_CUDA(cudaEventRecord(lane.tick_ev[slot], sst));
  std::lock_guard<std::mutex> lk(mu);
  stats.ticks += 1;
  stats.probe_slices += advanced;
  stats.launches += launched;
  stats.groups += (long long)started.size();
  stats.throttle_ms += ms_between(t0, t1);
  stats.issue_ms += ms_between(t1, Clock::now());
  return Status::Ok();
}

void totem_server::sched_loop() {
  cudaSetDevice(device);
  auto idle = [&] { return lanes[0]->planner.idle() && lanes[1]->planner.idle(); };
  for (;;) {
    std::vector<Request*> fresh;
    {
      std::unique_lock<std::mutex> lk(mu);
      const Clock::time_point w0 = Clock::now();
      cv.wait(lk, [&] { return !ready.empty() || !idle() || (stopping && prep_exited) || !fatal.ok(); });
      stats.idle_ms += ms_between(w0, Clock::now());
      if (!fatal.ok()) break;
      if (ready.empty() && idle() && stopping && prep_exited) break;
      while (!ready.empty()) {
        fresh.push_back(ready.front());
        ready.pop_front();
      }
      for (Request* r : fresh) {
        r->state = TOTEM_REQ_RUNNING;
        r->t_ready = Clock::now();
        running[r->ticket] = r;
      }
    }
    Status st;
    for (Request* r : fresh) {
      r->lane = (r->items * r->item_bytes <= lanes[0]->wave) ? 0 : 1;
      st = totem::cuda_status(cudaStreamWaitEvent(lanes[r->lane]->st, r->ready, 0), "cudaStreamWaitEvent");
      if (!st.ok()) break;
      if (r->items == 0) {
        st = complete_request(r);
        if (!st.ok()) break;
        continue;
      }
      totem::PlanRequest pr;
      pr.id = r->ticket;
      pr.n = r->sess->h;
      pr.items = r->items;
      pr.slices = r->sess->slices;
      pr.item_bytes = r->item_bytes;
      lanes[r->lane]->planner.add(pr);
    }
    for (auto& lane : lanes) {
      if (!st.ok() || lane->planner.idle()) continue;
      bool progressed = false;
      st = tick_once(*lane, &progressed);
      if (progressed) ++lane->tick;
    }
    if (!st.ok()) {
      fail_all(st);
      break;
    }
  }
  for (auto& lane : lanes) cudaStreamSynchronize(lane->st);
  std::lock_guard<std::mutex> lk(mu);
  sched_exited = true;
  cv.notify_all();
}

// ---------------------------------------------------------------------------------------------
// complete: results to the caller, retire device state
// ---------------------------------------------------------------------------------------------
void totem_server::done_loop() {
  cudaSetDevice(device);
  for (;;) {
    Request* r = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv.wait(lk, [&] { return !completing.empty() || (sched_exited && prep_exited); });
      if (completing.empty()) break;
      r = completing.front();
      completing.pop_front();
    }
    Status st = totem::cuda_status(cudaEventSynchronize(r->done), "cudaEventSynchronize");
    if (st.ok()) st = r->sess->download(&r->out);
    delete r->sess;
    r->sess = nullptr;
    for (cudaEvent_t* e : {&r->ready, &r->handoff, &r->done})
      if (*e) {
        cudaEventDestroy(*e);
        *e = nullptr;
      }
    std::lock_guard<std::mutex> lk(mu);
    static_used -= r->reserve;
    stats.requests_done += 1;
    if (st.ok()) {
      r->state = TOTEM_REQ_DONE;
      r->status = TOTEM_OK;
      r->t_done = Clock::now();
    } else {
      fail_request(r, st);
    }
    cv.notify_all();
  }
}

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------
namespace {

int server_fail(const Status& s) {
  totem::set_last_error(s.msg);
  return s.code;
}

void shutdown(totem_server* s) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    s->cv.notify_all();
  }
  for (auto& t : s->prep_thrs)
    if (t.joinable()) t.join();
  if (s->sched_thr.joinable()) s->sched_thr.join();
  if (s->done_thr.joinable()) s->done_thr.join();
  cudaSetDevice(s->device);
  for (auto& kv : s->reqs)
    if (kv.second->sess) {
      cudaStreamSynchronize(kv.second->sess->stream);
      delete kv.second->sess;
      kv.second->sess = nullptr;
    }
  s->tw.clear();
  for (auto& lane : s->lanes) {
    if (lane->st) cudaStreamSynchronize(lane->st);
    for (auto& e : lane->tick_ev)
      if (e) cudaEventDestroy(e);
    if (lane->h_stage) cudaFreeHost(lane->h_stage);
    if (lane->d_stage) cudaFree(lane->d_stage);
    if (lane->st) cudaStreamDestroy(lane->st);
  }
  s->lanes.clear();
  if (s->pool) {
    cudaDeviceSynchronize();
    cudaMemPoolDestroy(s->pool);
  }
}

}  // namespace

// Worker thread body.  A host exception (allocation failure) fails every pending request instead
// of terminating the caller's process; the worker then exits as on shutdown.
void run_worker(totem_server* s, int which) {
  try {
    if (which == 0) s->prep_loop();
    else if (which == 1) s->sched_loop();
    else s->done_loop();
  } catch (const std::exception& e) {
    s->fail_all(Status::Err(TOTEM_ERR_OOM, std::string("server worker: ") + e.what()));
    std::lock_guard<std::mutex> lk(s->mu);
    if (which == 0 && --s->prep_live == 0) s->prep_exited = true;
    if (which == 1) s->sched_exited = true;
    s->cv.notify_all();
  }
}

extern "C" {

int totem_server_create(const TotemServerOptions* opt, totem_server** out) {
  if (!out) return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "out is NULL"));
  *out = nullptr;
  TotemServerOptions o{};
  o.struct_size = (int)sizeof(TotemServerOptions);
  o.device = -1;
  if (opt) {
    if (opt->struct_size != (int)sizeof(TotemServerOptions))
      return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "TotemServerOptions.struct_size does not match this library"));
    o = *opt;
  }
  if (o.policy != TOTEM_SCHED_FIFO && o.policy != TOTEM_SCHED_SHORTEST)
    return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "unknown scheduling policy"));
  int dev = o.device;
  Status st = totem::pick_device(&dev);
  if (!st.ok()) return server_fail(st);
  std::unique_ptr<totem_server> s(new totem_server());
  s->device = dev;
  s->opt = o;
  st = s->init();
  if (!st.ok()) {
    shutdown(s.get());
    return server_fail(st);
  }
  totem_server* raw = s.get();
  // two preparation threads by default: with a mix up to 1024^2 windows (2048^2 potentials)
  // burst throughput was 218-221K probe*slices/s against 202-209K with one, and equal within
  // the run-to-run spread on 256^2/512^2 mixes; three were slower (concurrent uploads from
  // pageable memory contend: 52-177 ms per preparation against 16-31 ms with one thread)
  const int np = o.prep_threads > 0 ? o.prep_threads : 2;
  raw->prep_live = np;
  for (int i = 0; i < np; ++i) raw->prep_thrs.emplace_back(run_worker, raw, 0);
  raw->sched_thr = std::thread(run_worker, raw, 1);
  raw->done_thr = std::thread(run_worker, raw, 2);
  *out = s.release();
  return TOTEM_OK;
}

int totem_server_submit(totem_server* s, const TotemStemArgs* args, TotemStemOut* out, unsigned long long* ticket) {
  if (!s || !ticket) return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "NULL argument"));
  Status st = totem_session::validate(args, true);
  if (!st.ok()) return server_fail(st);
  if (args->depth > 0 && !fused_window(args->height, args->width))
    return server_fail(Status::Err(TOTEM_ERR_UNSUPPORTED,
                                   "the server runs square windows of 64..2048: powers of two or the mixed-radix edges"));
  if (args->depth > 0 && args->slices < 1)
    return server_fail(Status::Err(TOTEM_ERR_UNSUPPORTED, "the server needs at least one slice"));
  std::unique_ptr<Request> r(new Request());
  r->args = *args;
  if (out) r->out = *out;
  r->reserve = resident_bytes(*args);
  r->est = est_seconds(*args);
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->fatal.ok()) return server_fail(s->fatal);
  if (s->stopping) return server_fail(Status::Err(TOTEM_ERR_STATE, "server is shutting down"));
  r->ticket = s->next_ticket++;
  *ticket = r->ticket;
  s->submitted.push_back(r.get());
  s->reqs[r->ticket] = std::move(r);
  s->cv.notify_all();
  return TOTEM_OK;
}

int totem_server_wait(totem_server* s, unsigned long long ticket, int timeout_ms) {
  if (!s) return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "server is NULL"));
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "unknown ticket"));
  Request* r = it->second.get();
  auto finished = [&] { return r->state == TOTEM_REQ_DONE || r->state == TOTEM_REQ_FAILED; };
  if (timeout_ms < 0) s->cv.wait(lk, finished);
  else if (!s->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished))
    return server_fail(Status::Err(TOTEM_ERR_TIMEOUT, "request not finished"));
  if (r->status != TOTEM_OK) return server_fail(Status::Err(r->status, r->error));
  return TOTEM_OK;
}

int totem_server_info(totem_server* s, unsigned long long ticket, TotemRequestInfo* info) {
  if (!s || !info) return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "NULL argument"));
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "unknown ticket"));
  const Request* r = it->second.get();
  *info = TotemRequestInfo{};
  info->state = r->state;
  info->status = r->status;
  const bool done = r->state == TOTEM_REQ_DONE || r->state == TOTEM_REQ_FAILED;
  if (r->state >= TOTEM_REQ_PREPARING && r->t_admit != Clock::time_point()) info->queued_ms = ms_between(r->t_submit, r->t_admit);
  if (r->t_ready != Clock::time_point()) info->prepare_ms = ms_between(r->t_admit, r->t_ready);
  if (done && r->t_ready != Clock::time_point()) info->run_ms = ms_between(r->t_ready, r->t_done);
  if (done) info->latency_ms = ms_between(r->t_submit, r->t_done);
  info->probe_slices = (long long)r->args.w_num * r->args.depth * r->args.slices;
  if (r->state == TOTEM_REQ_FAILED) totem::set_last_error(r->error);
  return TOTEM_OK;
}

int totem_server_stats(totem_server* s, TotemServerStats* out) {
  if (!s || !out) return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "NULL argument"));
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  return TOTEM_OK;
}

int totem_server_destroy(totem_server* s) {
  if (!s) return TOTEM_OK;
  shutdown(s);
  delete s;
  return TOTEM_OK;
}

int totem_plan_simulate(int count, const int* n, const long long* items, const int* slices, const int* arrive,
                        unsigned long long wave_bytes, unsigned long long chunk_bytes, int policy, int* first_tick,
                        int* done_tick, unsigned long long* max_inflight) {
  if (count < 0 || (count > 0 && (!n || !items || !slices || !arrive || !first_tick || !done_tick)) || !max_inflight)
    return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "NULL argument"));
  if (policy != TOTEM_SCHED_FIFO && policy != TOTEM_SCHED_SHORTEST)
    return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "unknown scheduling policy"));
  if (wave_bytes == 0) return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "wave_bytes is 0"));
  std::vector<int> order(count);
  std::vector<long long> left(count);
  for (int i = 0; i < count; ++i) {
    if (n[i] <= 0 || items[i] < 0 || slices[i] < 1 || arrive[i] < 0)
      return server_fail(Status::Err(TOTEM_ERR_INVALID_ARG, "request sizes out of range"));
    order[i] = i;
    left[i] = items[i];
    first_tick[i] = done_tick[i] = -1;
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return arrive[a] < arrive[b]; });
  totem::Planner planner(wave_bytes, chunk_bytes ? chunk_bytes : wave_bytes / 4, policy, 4096);
  *max_inflight = 0;
  size_t added = 0;
  int remaining = count;
  for (long long tick = 0; remaining > 0; ++tick) {
    if (tick > (1ll << 30)) return server_fail(Status::Err(TOTEM_ERR_STATE, "simulation does not terminate"));
    while (added < order.size() && arrive[order[added]] <= tick) {
      const int i = order[added++];
      if (items[i] == 0) {
        first_tick[i] = done_tick[i] = (int)tick;
        --remaining;
        continue;
      }
      totem::PlanRequest r;
      r.id = (unsigned long long)i;
      r.n = n[i];
      r.items = items[i];
      r.slices = slices[i];
      r.item_bytes = (size_t)n[i] * n[i] * sizeof(float2);
      planner.add(r);
    }
    for (const totem::PlanGroup& g : planner.start((int)tick))
      if (first_tick[g.req] < 0) first_tick[g.req] = (int)tick;
    *max_inflight = std::max<unsigned long long>(*max_inflight, planner.inflight());
    for (const totem::PlanGroup& g : planner.finish((int)tick)) {
      left[g.req] -= g.items;
      if (left[g.req] == 0) {
        done_tick[g.req] = (int)tick;
        --remaining;
      }
    }
  }
  return TOTEM_OK;
}

}  // extern "C"
