// server.cu -- continuous-batching request server (gb2_server_*).
//
// A request is a batch of pairs, each Smith-Waterman or WFA.  Requests queue
// in arrival order.  A scheduler thread admits the oldest ones while the
// device memory they need fits the HBM budget, gathers them into a group and
// launches the group on one of the server's executors (its own stream,
// planning buffers and scratch) as soon as an executor is free; with several
// executors, groups formed from later arrivals run while earlier groups are
// still on the GPU.  A host callback on the executor's stream marks the
// group finished; the scheduler then copies each request's results into the
// caller's arrays and wakes its waiter.  Every pair of a group runs through
// the same sw_core / wfa_core as the blocking entry points, so a result does
// not depend on what else is in flight.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>

#include "runtime.cuh"

using namespace gb2;

namespace {

using Clock = std::chrono::steady_clock;

constexpr int64_t kAlign = 256;
inline int64_t align_up(int64_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }

struct Req {
    uint64_t ticket = 0;
    gb2_request r{};
    int64_t n_sw = 0, n_wfa = 0;
    int64_t sw_qw = 0, sw_rw = 0, wfa_qw = 0, wfa_rw = 0;  // packed words per side
    int64_t sw_qmax = 0, sw_rmax = 0, wfa_qmax = 0, wfa_rmax = 0;
    int32_t max_band = 0;
    int64_t need_alone = 0;             // device bytes of a group holding only this request
    int64_t sw_base = 0, wfa_base = 0;  // first index in the group's result arrays
    Clock::time_point t_submit, t_done;
    int status = 1;  // 1 queued, 2 running, 0 done, < 0 failed
};

struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
    // buffers outgrown while the server runs: freed when it stops, because
    // cudaFreeHost waits for the device, which would stall the groups running
    // on the other slots
    std::vector<void *> retired;
};

int ensure_host(HostBuf &b, size_t bytes)
{
    if (bytes <= b.cap)
        return GB2_OK;
    if (b.p)
        b.retired.push_back(b.p);
    b.p = nullptr;
    b.cap = 0;
    // pinning memory is slow: grow with headroom, rarely
    const size_t cap = std::max<size_t>(2 * bytes, 1 << 20);
    if (pinned_alloc(&b.p, cap) != cudaSuccess) {
        cudaGetLastError();
        return GB2_ENOMEM;
    }
    b.cap = cap;
    return GB2_OK;
}

// Byte layout of one group's input and output staging.
struct Layout {
    int64_t n_sw = 0, n_wfa = 0, sw_qw = 0, sw_rw = 0, wfa_qw = 0, wfa_rw = 0;
    int64_t sw_qmax = 0, sw_rmax = 0, wfa_qmax = 0, wfa_rmax = 0;
    int32_t max_band = 0;
    // input sections
    int64_t o_sqw, o_srw, o_sqo, o_sql, o_sro, o_srl, o_band, o_wqw, o_wrw, o_wqo, o_wql, o_wro,
        o_wrl, in_bytes;
    // output sections
    int64_t o_sout, o_wout, o_flag, out_bytes;

    void finish()
    {
        int64_t o = 0;
        auto take = [&](int64_t bytes) {
            const int64_t at = o;
            o = align_up(o + std::max<int64_t>(bytes, 8));
            return at;
        };
        o_sqw = take(sw_qw * 8);
        o_srw = take(sw_rw * 8);
        o_sqo = take(n_sw * 8);
        o_sql = take(n_sw * 8);
        o_sro = take(n_sw * 8);
        o_srl = take(n_sw * 8);
        o_band = take(n_sw * 4);
        o_wqw = take(wfa_qw * 8);
        o_wrw = take(wfa_rw * 8);
        o_wqo = take(n_wfa * 8);
        o_wql = take(n_wfa * 8);
        o_wro = take(n_wfa * 8);
        o_wrl = take(n_wfa * 8);
        in_bytes = o;
        o = 0;
        o_sout = take(n_sw * (int64_t)sizeof(gb2_sw_result));
        o_wout = take(n_wfa * 4);
        o_flag = take(16);
        out_bytes = o;
    }
};

struct Slot;
struct CallbackArg {
    gb2_server *srv;
    Slot *slot;
};

struct Slot {
    Exec x;
    DevBuf d_in, d_out;
    HostBuf h_in, h_out;
    bool busy = false;
    bool finished = false;
    int rc = GB2_OK;
    std::vector<Req *> reqs;
    Layout lay;
    int64_t bytes = 0;
    CallbackArg cb{};
};

}  // namespace

struct gb2_server {
    gb2_ctx *c = nullptr;
    gb2_server_cfg cfg{};
    std::vector<std::unique_ptr<Slot>> slots;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<Req *> pending;
    std::map<uint64_t, Req *> table;
    uint64_t next_ticket = 1;
    bool stopping = false;
    bool hold = false;  // admission held (gb2_server_hold)
    std::thread th;
    gb2_server_stats st{};
    // device memory pool of the slots' buffers: they grow by stream-ordered
    // allocation, so a slot meeting a larger group than before does not stall
    // the groups running on the other slots (cudaFree would synchronise the
    // device); freed memory stays in the pool
    cudaMemPool_t pool = nullptr;
};

namespace {

int gcd_i(int a, int b)
{
    while (b) {
        const int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// Device bytes one group of the given shape holds: staging copies, results,
// planning arrays, literal-kernel rows and WFA rings.
int64_t group_bytes(const Layout &l, const gb2_wfa_cfg &w, int sm_count)
{
    int64_t b = align_up(l.in_bytes) + align_up(l.out_bytes);
    b += l.n_sw * 8 + (int64_t)kSwClasses * kLenBuckets * 4 + 8192;  // keys, queue, counts
    if (l.n_sw) {
        const int64_t lit_grid = std::min<int64_t>((l.n_sw + 127) / 128, (int64_t)sm_count * 2);
        b += lit_grid * 128 * 3 * (2 * (int64_t)l.max_band + 1) * 8;
    }
    if (l.n_wfa) {
        const int g = gcd_i(w.x, gcd_i(w.o, w.e));
        const int64_t nslot = std::max(w.x / g, (w.o + w.e) / g) + 1 + 2 * (w.e / g + 1);
        // the single-kernel design (tuning variants): rings per warp in flight
        const int64_t warps = std::min<int64_t>(l.n_wfa + 3, (int64_t)sm_count * 16);
        const int64_t rings =
            warps * nslot * (((l.wfa_qmax + l.wfa_rmax + 5) + 31) & ~int64_t(31)) * 4;
        // the tiers: their queues, the suspended pairs' records of the two
        // transitions, and the G tier's per-block rings
        const WfaTierPlan pl = wfa_tier_plan(WfaParams{w.x, w.o, w.e, w.max_error},
                                             l.wfa_qmax, l.wfa_rmax);
        int64_t tiers = l.n_wfa * (8 * kWfaShared + 4) + (int64_t)sm_count * pl.gring_block_bytes;
        for (int t = 0; t + 1 < kWfaShared; ++t)
            tiers += std::min<int64_t>(l.n_wfa, kTierDumpCap / pl.dump_stride[t]) *
                     pl.dump_stride[t];
        b += std::max(rings, tiers);
        b += l.n_wfa * 8 + kLenBuckets * 4;
    }
    return b;
}

void add_req(Layout &l, const Req &q)
{
    l.n_sw += q.n_sw;
    l.n_wfa += q.n_wfa;
    l.sw_qw += q.sw_qw;
    l.sw_rw += q.sw_rw;
    l.wfa_qw += q.wfa_qw;
    l.wfa_rw += q.wfa_rw;
    l.sw_qmax = std::max(l.sw_qmax, q.sw_qmax);
    l.sw_rmax = std::max(l.sw_rmax, q.sw_rmax);
    l.wfa_qmax = std::max(l.wfa_qmax, q.wfa_qmax);
    l.wfa_rmax = std::max(l.wfa_rmax, q.wfa_rmax);
    l.max_band = std::max(l.max_band, q.max_band);
}

bool same_cfg(const gb2_request &a, const gb2_request &b)
{
    return memcmp(&a.sw_cfg, &b.sw_cfg, sizeof a.sw_cfg) == 0 &&
           memcmp(&a.wfa_cfg, &b.wfa_cfg, sizeof a.wfa_cfg) == 0;
}

void CUDART_CB on_group_done(void *p)
{
    CallbackArg *a = (CallbackArg *)p;
    {
        std::lock_guard<std::mutex> lk(a->srv->mu);
        a->slot->finished = true;
    }
    a->srv->cv_sched.notify_one();
}

// Copies the group's pairs from the callers' arrays into pinned staging,
// uploads them, runs the kernels and queues the result copy and the
// completion callback.  Runs without the server lock.
int launch_group(gb2_server *s, Slot &sl)
{
    gb2_ctx *c = s->c;
    Exec &x = sl.x;
    Layout &L = sl.lay;
    int rc;
    if ((rc = ensure_host(sl.h_in, L.in_bytes)) || (rc = ensure_host(sl.h_out, L.out_bytes)))
        return rc;
    char *h = (char *)sl.h_in.p;
    uint64_t *sqw = (uint64_t *)(h + L.o_sqw), *srw = (uint64_t *)(h + L.o_srw);
    int64_t *sqo = (int64_t *)(h + L.o_sqo), *sql = (int64_t *)(h + L.o_sql);
    int64_t *sro = (int64_t *)(h + L.o_sro), *srl = (int64_t *)(h + L.o_srl);
    int32_t *band = (int32_t *)(h + L.o_band);
    uint64_t *wqw = (uint64_t *)(h + L.o_wqw), *wrw = (uint64_t *)(h + L.o_wrw);
    int64_t *wqo = (int64_t *)(h + L.o_wqo), *wql = (int64_t *)(h + L.o_wql);
    int64_t *wro = (int64_t *)(h + L.o_wro), *wrl = (int64_t *)(h + L.o_wrl);
    int64_t is = 0, iw = 0, sq = 0, sr = 0, wq = 0, wr = 0;
    for (Req *rq : sl.reqs) {
        const gb2_request &R = rq->r;
        rq->sw_base = is;
        rq->wfa_base = iw;
        for (int64_t i = 0; i < R.n_pairs; ++i) {
            const int64_t ql = R.q_lengths[i], rl = R.r_lengths[i];
            const int64_t nq = words_for(ql), nr = words_for(rl);
            const bool wfa = R.kinds && R.kinds[i] == 1;
            if (!wfa) {
                memcpy(sqw + sq, R.q_packed + R.q_offsets[i], (size_t)nq * 8);
                memcpy(srw + sr, R.r_packed + R.r_offsets[i], (size_t)nr * 8);
                sqo[is] = sq;
                sql[is] = ql;
                sro[is] = sr;
                srl[is] = rl;
                band[is] = R.bands ? R.bands[i] : R.sw_cfg.band_width;
                sq += nq;
                sr += nr;
                ++is;
            } else {
                memcpy(wqw + wq, R.q_packed + R.q_offsets[i], (size_t)nq * 8);
                memcpy(wrw + wr, R.r_packed + R.r_offsets[i], (size_t)nr * 8);
                wqo[iw] = wq;
                wql[iw] = ql;
                wro[iw] = wr;
                wrl[iw] = rl;
                wq += nq;
                wr += nr;
                ++iw;
            }
        }
    }
    if ((rc = ensure(c, sl.d_in, L.in_bytes, x.st)) || (rc = ensure(c, sl.d_out, L.out_bytes, x.st)))
        return rc;
    GB2_CU(c, cudaMemcpyAsync(sl.d_in.p, sl.h_in.p, L.in_bytes, cudaMemcpyHostToDevice, x.st));
    char *d = (char *)sl.d_in.p;
    char *dout = (char *)sl.d_out.p;
    const gb2_request &R0 = sl.reqs.front()->r;
    const int flags = s->cfg.flags | GB2_FLAG_BATCHED;
    if (L.n_sw) {
        SeqView qv{(const uint64_t *)(d + L.o_sqw), (const int64_t *)(d + L.o_sqo),
                   (const int64_t *)(d + L.o_sql), 0, std::max<int64_t>(L.sw_qw, 1)};
        SeqView rv{(const uint64_t *)(d + L.o_srw), (const int64_t *)(d + L.o_sro),
                   (const int64_t *)(d + L.o_srl), 0, std::max<int64_t>(L.sw_rw, 1)};
        // bands come per pair from the staged array; the config's own band is unused
        gb2_sw_cfg cfg = R0.sw_cfg;
        cfg.band_width = L.max_band;
        SwPlanInfo pi;
        if ((rc = sw_validate(c, &cfg, nullptr, 0, L.sw_qmax, L.sw_rmax, pi)))
            return rc;
        pi.uniform_band = false;
        pi.max_band = L.max_band;
        if ((rc = sw_core(c, x, qv, rv, L.sw_qmax, L.sw_rmax, &cfg,
                          (const int32_t *)(d + L.o_band), pi, L.n_sw,
                          (gb2_sw_result *)(dout + L.o_sout), flags)))
            return rc;
    }
    if (L.n_wfa) {
        SeqView qv{(const uint64_t *)(d + L.o_wqw), (const int64_t *)(d + L.o_wqo),
                   (const int64_t *)(d + L.o_wql), 0, std::max<int64_t>(L.wfa_qw, 1)};
        SeqView rv{(const uint64_t *)(d + L.o_wrw), (const int64_t *)(d + L.o_wro),
                   (const int64_t *)(d + L.o_wrl), 0, std::max<int64_t>(L.wfa_rw, 1)};
        if ((rc = wfa_begin(c, x)) ||
            (rc = wfa_core(c, x, qv, rv, L.wfa_qmax, L.wfa_rmax, &R0.wfa_cfg, L.n_wfa,
                           (int32_t *)(dout + L.o_wout), flags)))
            return rc;
        GB2_CU(c, cudaMemcpyAsync(dout + L.o_flag, x.errflag.p, 4, cudaMemcpyDeviceToDevice,
                                  x.st));
    } else {
        GB2_CU(c, cudaMemsetAsync(dout + L.o_flag, 0, 4, x.st));
    }
    GB2_CU(c, cudaMemcpyAsync(sl.h_out.p, sl.d_out.p, L.out_bytes, cudaMemcpyDeviceToHost, x.st));
    sl.cb = CallbackArg{s, &sl};
    GB2_CU(c, cudaLaunchHostFunc(x.st, on_group_done, &sl.cb));
    return GB2_OK;
}

// Hands a finished group's results to its requests.  Server lock held.
void complete_group(gb2_server *s, Slot &sl)
{
    if (sl.rc != GB2_OK)  // a failed launch may have left work queued on the stream
        cudaStreamSynchronize(sl.x.st);
    const Layout &L = sl.lay;
    const char *h = (const char *)sl.h_out.p;
    const gb2_sw_result *sout = (const gb2_sw_result *)(h + L.o_sout);
    const int32_t *wout = (const int32_t *)(h + L.o_wout);
    int flag = 0;
    if (sl.rc == GB2_OK)
        memcpy(&flag, h + L.o_flag, 4);
    const int status = sl.rc != GB2_OK ? sl.rc : (flag ? GB2_EKERNEL : GB2_OK);
    const Clock::time_point now = Clock::now();
    for (Req *rq : sl.reqs) {
        if (status == GB2_OK) {
            const gb2_request &R = rq->r;
            int64_t is = rq->sw_base, iw = rq->wfa_base;
            for (int64_t i = 0; i < R.n_pairs; ++i) {
                if (R.kinds && R.kinds[i] == 1)
                    R.wfa_out[i] = wout[iw++];
                else
                    R.sw_out[i] = sout[is++];
            }
            s->st.completed += 1;
            s->st.pairs_completed += R.n_pairs;
        } else {
            s->st.failed += 1;
        }
        rq->status = status;
        rq->t_done = now;
    }
    s->st.inflight_bytes -= sl.bytes;
    sl.reqs.clear();
    sl.busy = false;
    sl.finished = false;
    sl.rc = GB2_OK;
}

void scheduler(gb2_server *s)
{
    cudaSetDevice(s->c->device);
    const int64_t max_pairs = s->cfg.max_group_pairs > 0 ? s->cfg.max_group_pairs : 65536;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progressed = false;
        for (auto &up : s->slots) {
            Slot &sl = *up;
            if (sl.busy && sl.finished) {
                complete_group(s, sl);
                progressed = true;
            }
        }
        if (progressed)
            s->cv_done.notify_all();
        // launch groups while an executor is free and the oldest request fits
        for (auto &up : s->slots) {
            Slot &sl = *up;
            if (sl.busy || s->pending.empty() || s->hold)
                continue;
            Layout L;
            std::vector<Req *> take;
            const gb2_request &head = s->pending.front()->r;
            for (auto it = s->pending.begin(); it != s->pending.end();) {
                Req *rq = *it;
                if (!same_cfg(rq->r, head)) {
                    ++it;
                    continue;
                }
                Layout T = L;
                add_req(T, *rq);
                T.finish();
                const int64_t need = group_bytes(T, head.wfa_cfg, s->c->sm_count);
                const int64_t pairs = T.n_sw + T.n_wfa;
                if ((!take.empty() && pairs > max_pairs) ||
                    s->st.inflight_bytes + need > s->cfg.hbm_budget_bytes)
                    break;  // requests keep their arrival order: stop at the first misfit
                L = T;
                take.push_back(rq);
                it = s->pending.erase(it);
            }
            if (take.empty())
                break;  // the oldest request waits for memory to free up
            L.finish();
            sl.lay = L;
            sl.reqs = take;
            sl.bytes = group_bytes(L, head.wfa_cfg, s->c->sm_count);
            sl.busy = true;
            sl.finished = false;
            for (Req *rq : take)
                rq->status = 2;
            s->st.inflight_bytes += sl.bytes;
            s->st.peak_inflight_bytes = std::max(s->st.peak_inflight_bytes, s->st.inflight_bytes);
            s->st.groups_launched += 1;
            lk.unlock();
            const int rc = launch_group(s, sl);
            lk.lock();
            if (rc != GB2_OK) {
                sl.rc = rc;
                sl.finished = true;
            }
        }
        bool any_busy = false;
        for (auto &up : s->slots)
            any_busy |= up->busy;
        if (s->stopping && s->pending.empty() && !any_busy)
            break;
        // sleep until a group finishes, or a free executor can take the
        // oldest request (it fits the budget), or a stop finds nothing left
        s->cv_sched.wait(lk, [&] {
            bool busy = false, free_slot = false;
            for (auto &up : s->slots) {
                if (up->busy && up->finished)
                    return true;
                busy |= up->busy;
                free_slot |= !up->busy;
            }
            if (free_slot && !s->pending.empty() && !s->hold &&
                s->st.inflight_bytes + s->pending.front()->need_alone <= s->cfg.hbm_budget_bytes)
                return true;
            return s->stopping && s->pending.empty() && !busy;
        });
    }
}

}  // namespace

extern "C" {

int gb2_server_start(gb2_ctx *c, const gb2_server_cfg *cfg, gb2_server **out)
{
    if (!c || !cfg || !out)
        return GB2_EINVAL;
    *out = nullptr;
    if (cfg->max_inflight_groups < 1 || cfg->max_inflight_groups > 8 ||
        cfg->hbm_budget_bytes <= 0 || cfg->max_group_pairs < 0)
        return set_err(c, GB2_EINVAL, "server config out of range");
    cudaSetDevice(c->device);
    gb2_server *s = new gb2_server();
    s->c = c;
    s->cfg = *cfg;
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = c->device;
        uint64_t keep = UINT64_MAX;
        if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess ||
            cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep) !=
                cudaSuccess) {
            cudaGetLastError();  // without a pool the slots grow with cudaMalloc
            if (s->pool)
                cudaMemPoolDestroy(s->pool);
            s->pool = nullptr;
        }
    }
    for (int i = 0; i < cfg->max_inflight_groups; ++i) {
        auto sl = std::make_unique<Slot>();
        for (DevBuf *b : {&sl->d_in, &sl->d_out, &sl->x.keys, &sl->x.queue, &sl->x.counts,
                          &sl->x.seg, &sl->x.counters, &sl->x.scratch64, &sl->x.scratch32,
                          &sl->x.work, &sl->x.errflag, &sl->x.tierq, &sl->x.dumps,
                          &sl->x.ubound})
            b->pool = s->pool;
        if (exec_init(sl->x) != GB2_OK) {
            exec_free(sl->x);
            for (auto &o : s->slots)
                exec_free(o->x);
            if (s->pool)
                cudaMemPoolDestroy(s->pool);
            delete s;
            return set_err(c, GB2_ECUDA, "creating a server executor failed");
        }
        s->slots.push_back(std::move(sl));
    }
    s->th = std::thread(scheduler, s);
    *out = s;
    return GB2_OK;
}

int gb2_server_submit(gb2_server *s, const gb2_request *req, uint64_t *ticket)
{
    if (!s || !req || !ticket)
        return GB2_EINVAL;
    gb2_ctx *c = s->c;
    const int64_t n = req->n_pairs;
    if (n < 0 || (n > 0 && (!req->q_packed || !req->q_offsets || !req->q_lengths ||
                            !req->r_packed || !req->r_offsets || !req->r_lengths)))
        return set_err(c, GB2_EINVAL, "request arrays missing");
    Req *rq = new Req();
    rq->r = *req;
    int rc = GB2_OK;
    for (int64_t i = 0; i < n && rc == GB2_OK; ++i) {
        const int64_t ql = req->q_lengths[i], rl = req->r_lengths[i];
        if (ql < 0 || rl < 0 || req->q_offsets[i] < 0 || req->r_offsets[i] < 0) {
            rc = set_err(c, GB2_EINVAL, "negative offset or length in request pair %lld",
                         (long long)i);
            break;
        }
        const bool wfa = req->kinds && req->kinds[i] == 1;
        if (req->kinds && req->kinds[i] != 0 && req->kinds[i] != 1)
            rc = set_err(c, GB2_EINVAL, "pair kind must be 0 (SW) or 1 (WFA)");
        if (wfa) {
            rq->n_wfa++;
            rq->wfa_qw += words_for(ql);
            rq->wfa_rw += words_for(rl);
            rq->wfa_qmax = std::max(rq->wfa_qmax, ql);
            rq->wfa_rmax = std::max(rq->wfa_rmax, rl);
        } else {
            const int32_t b = req->bands ? req->bands[i] : req->sw_cfg.band_width;
            if (b < 0)
                rc = set_err(c, GB2_EINVAL, "negative band in request pair %lld", (long long)i);
            rq->n_sw++;
            rq->sw_qw += words_for(ql);
            rq->sw_rw += words_for(rl);
            rq->sw_qmax = std::max(rq->sw_qmax, ql);
            rq->sw_rmax = std::max(rq->sw_rmax, rl);
            rq->max_band = std::max(rq->max_band, b);
        }
    }
    if (rc == GB2_OK && rq->n_sw > 0) {
        SwPlanInfo pi;
        gb2_sw_cfg cfg = req->sw_cfg;
        cfg.band_width = rq->max_band;
        if (!req->sw_out)
            rc = set_err(c, GB2_EINVAL, "sw_out is NULL");
        else
            rc = sw_validate(c, &cfg, nullptr, 0, rq->sw_qmax, rq->sw_rmax, pi);
    }
    if (rc == GB2_OK && rq->n_wfa > 0) {
        if (!req->wfa_out)
            rc = set_err(c, GB2_EINVAL, "wfa_out is NULL");
        else if ((rc = wfa_validate(c, &req->wfa_cfg, rq->n_wfa)) == GB2_OK &&
                 (rq->wfa_qmax >= (1ll << 30) || rq->wfa_rmax >= (1ll << 30)))
            rc = set_err(c, GB2_ERANGE, "sequence longer than 2^30");
    }
    if (rc == GB2_OK) {
        Layout L;
        add_req(L, *rq);
        L.finish();
        rq->need_alone = group_bytes(L, req->wfa_cfg, c->sm_count);
        if (rq->need_alone > s->cfg.hbm_budget_bytes)
            rc = set_err(c, GB2_ENOMEM, "request needs more device memory than the budget");
    }
    if (rc != GB2_OK) {
        delete rq;
        return rc;
    }
    rq->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) {
            delete rq;
            return GB2_ESTATE;
        }
        rq->ticket = s->next_ticket++;
        s->table[rq->ticket] = rq;
        s->st.submitted += 1;
        if (n == 0) {
            rq->status = GB2_OK;
            rq->t_done = rq->t_submit;
        } else {
            s->pending.push_back(rq);
        }
        *ticket = rq->ticket;
    }
    s->cv_sched.notify_one();
    return GB2_OK;
}

int gb2_server_poll(gb2_server *s, uint64_t ticket, int *done)
{
    if (!s || !done)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->table.find(ticket);
    if (it == s->table.end())
        return GB2_EINVAL;
    *done = it->second->status <= 0 ? 1 : 0;
    return GB2_OK;
}

int gb2_server_wait(gb2_server *s, uint64_t ticket, int timeout_ms, double *latency_ms)
{
    if (!s)
        return GB2_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->table.find(ticket);
    if (it == s->table.end())
        return GB2_EINVAL;
    Req *rq = it->second;
    auto ready = [&] { return rq->status <= 0; };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
        return GB2_ETIMEOUT;
    if (latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(rq->t_done - rq->t_submit).count();
    const int status = rq->status;
    s->table.erase(it);
    delete rq;
    return status;
}

int gb2_server_stats_get(gb2_server *s, gb2_server_stats *st)
{
    if (!s || !st)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->st;
    return GB2_OK;
}

int gb2_server_hold(gb2_server *s, int hold)
{
    if (!s)
        return GB2_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping)
            return GB2_ESTATE;
        s->hold = hold != 0;
    }
    s->cv_sched.notify_one();
    return GB2_OK;
}

int gb2_server_cancel(gb2_server *s, uint64_t ticket)
{
    if (!s)
        return GB2_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->table.find(ticket);
        if (it == s->table.end())
            return GB2_EINVAL;
        Req *rq = it->second;
        if (rq->status != 1)
            return GB2_ESTATE;  // running or done
        for (auto p = s->pending.begin(); p != s->pending.end(); ++p)
            if (*p == rq) {
                s->pending.erase(p);
                break;
            }
        rq->status = GB2_ECANCELED;
        rq->t_done = Clock::now();
        s->st.cancelled += 1;
    }
    s->cv_done.notify_all();
    s->cv_sched.notify_one();  // the next queued request may fit now
    return GB2_OK;
}

int gb2_server_stop(gb2_server *s)
{
    if (!s)
        return GB2_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->hold = false;  // stopping finishes every queued request
    }
    s->cv_sched.notify_all();
    if (s->th.joinable())
        s->th.join();
    cudaSetDevice(s->c->device);
    for (auto &up : s->slots) {
        Slot &sl = *up;
        exec_free(sl.x);
        if (sl.d_in.p)
            cudaFree(sl.d_in.p);
        if (sl.d_out.p)
            cudaFree(sl.d_out.p);
        for (HostBuf *hb : {&sl.h_in, &sl.h_out}) {
            if (hb->p)
                cudaFreeHost(hb->p);
            for (void *p : hb->retired)
                cudaFreeHost(p);
        }
    }
    if (s->pool)
        cudaMemPoolDestroy(s->pool);
    for (auto &kv : s->table)
        delete kv.second;
    delete s;
    return GB2_OK;
}

}  // extern "C"
