// Serving loop: continuous batching of refactor+solve requests.
//
// Threads: callers (submit / poll), analysis threads (host COLAMD +
// pivoting factorization of new patterns, then the device upload; several
// new patterns are analysed at once), one scheduler thread (launches and
// completions).  The server's threads work on the device that was current
// when it was created.  Each stream owns a device
// arena and a pinned staging area; a launch bump-allocates all of its
// systems in the arena, so nothing is allocated on the device per request.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "luspice_b200.h"
#include "engine_internal.h"

namespace lusp {
namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

enum PatState { PAT_PENDING = 0, PAT_READY = 1, PAT_FAILED = 2 };

struct PatternEntry {
    uint64_t key = 0;
    int n = 0;
    std::vector<int> Ap, Ai;
    std::vector<double> Ax;        // values used to decide pivots
    PatternObj* pat = nullptr;
    int state = PAT_PENDING;
    int fail_rc = LUSP_OK;
    int users = 0;                 // requests referencing it
    long long last_use = 0;
    bool own = false;              // pivots chosen for one request's values:
                                   // never matched by a lookup
    // Escalation memory (a dynamic trial per pattern, not a condition
    // estimate): after two mixed requests in a row escalated, new requests
    // of the pattern start on the fp64 factor + GMRES-IR path, and every
    // kTrialEvery-th tries the mixed path again; a trial that succeeds
    // without escalation returns the pattern to the mixed path.
    int esc_run = 0;
    bool promoted = false;
    int since_trial = 0;
};
constexpr int kTrialEvery = 16;

// Requests are batched with others of their size class only, so a launch of
// small systems never waits for a system hundreds of times larger.
int size_class(int n) { return n < 2048 ? 0 : n < 12288 ? 1 : 2; }
// Launch cap of the large class: few enough systems that each is spread
// over several SMs (spread mode) instead of one 2-SM cluster.
constexpr int kLargeBatch = 8;

// MODE_FP64: the plain fp64 path (direct solve), for a server created in
// fp64; MODE_FP64_IR: a failed mixed system once more with an fp64 factor
// and GMRES-IR (the ladder's P-safe rung, run as its own launch).
enum Mode { MODE_MIXED = 0, MODE_MIXED_INNER64 = 1, MODE_FP64 = 2, MODE_FP64_IR = 3 };
static bool fp64_mode(int m) { return m == MODE_FP64 || m == MODE_FP64_IR; }

struct Request {
    long long id = 0;
    int n = 0;
    std::vector<double> vals, rhs, x;
    PatternEntry* pe = nullptr;
    int mode = MODE_MIXED;
    bool cache_hit = false;
    bool escalated = false;
    bool repivoted = false;        // analysed again with its own values
    bool trial = false;            // a mixed trial of a promoted pattern
    bool learned = false;          // its mixed attempt has updated the pattern's memory
    bool done = false;
    Clock::time_point t_submit, t_launch, t_done;
    lusp_serve_result res{};
};

struct Flight {
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    char* stage = nullptr;          // pinned: [values | rhs] up, [x | stats] down
    size_t stage_bytes = 0;
    bool busy = false;
    int cls = -1;                   // size class of the launch in flight
    std::vector<Request*> reqs;
    std::vector<size_t> x_off;      // per request, doubles into the download x area
    size_t down_x = 0, down_stats = 0;
};

uint64_t structure_hash(int n, const int* Ap, const int* Ai) { return pattern_hash(n, Ap, Ai, nullptr); }

}  // namespace

struct ServerObj {
    lusp_server_opts opts{};
    std::mutex mu;
    std::condition_variable cv_sched, cv_done, cv_analysis;
    bool stopping = false;
    long long next_id = 0;
    long long clock = 0;
    std::unordered_map<long long, std::unique_ptr<Request>> reqs;
    std::deque<Request*> queue;                       // waiting for a launch
    std::unordered_multimap<uint64_t, std::unique_ptr<PatternEntry>> patterns;
    std::deque<PatternEntry*> analysis_q;
    // Device patterns to free.  cudaFree waits for the whole device, so they
    // are freed only when no launch is in flight (the scheduler, idle).
    std::vector<PatternObj*> to_free;
    std::vector<Flight> flights;
    size_t pattern_bytes = 0, pattern_budget = 0;
    lusp_server_stats stats{};
    std::thread sched;
    std::vector<std::thread> analysis;               // host analysis of new patterns
    int device = 0;                                  // the device the server was created on

    int init();
    void shutdown();
    void analysis_loop();
    void sched_loop();
    bool try_launch(Flight& f);
    void complete(Flight& f);
    void evict_if_needed();
    void release(PatternEntry* pe);
};

int ServerObj::init() {
    cudaGetDevice(&device);
    // Every kernel a request may need (the fp64 rungs included) is loaded
    // before the first request, not in the middle of the stream.
    int prc = preload_kernels();
    if (prc != LUSP_OK) return prc;
    const int ns = std::max(1, opts.streams);
    flights.resize(ns);
    const size_t arena = (size_t)(opts.arena_gb * 1e9);
    const size_t stage = (size_t)(opts.staging_mb * 1e6);
    for (auto& f : flights) {
        cudaError_t e = cudaStreamCreateWithFlags(&f.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&f.ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&f.ev1);
        if (e == cudaSuccess) e = cudaMalloc(&f.arena, arena);
        if (e == cudaSuccess) e = cudaMallocHost(&f.stage, stage);
        if (e != cudaSuccess) return cuda_fail(e, "server_create");
        f.arena_bytes = arena;
        f.stage_bytes = stage;
    }
    const double budget = opts.hbm_budget_gb * 1e9 - (double)arena * ns;
    pattern_budget = budget > 0 ? (size_t)budget : 0;
    const int na = opts.analysis_threads > 0 ? opts.analysis_threads : 4;
    for (int t = 0; t < na; t++) analysis.emplace_back([this] { analysis_loop(); });
    sched = std::thread([this] { sched_loop(); });
    return LUSP_OK;
}

void ServerObj::shutdown() {
    {
        std::unique_lock<std::mutex> lk(mu);
        // Let queued and in-flight work finish.
        cv_done.wait(lk, [this] {
            if (!queue.empty()) return false;
            for (auto& f : flights)
                if (f.busy) return false;
            return analysis_q.empty();
        });
        stopping = true;
    }
    cv_sched.notify_all();
    cv_analysis.notify_all();
    if (sched.joinable()) sched.join();
    for (auto& t : analysis)
        if (t.joinable()) t.join();
    for (auto& f : flights) {
        if (f.st) cudaStreamSynchronize(f.st);
        if (f.arena) cudaFree(f.arena);
        if (f.stage) cudaFreeHost(f.stage);
        if (f.ev0) cudaEventDestroy(f.ev0);
        if (f.ev1) cudaEventDestroy(f.ev1);
        if (f.st) cudaStreamDestroy(f.st);
    }
    for (auto& kv : patterns)
        if (kv.second->pat) pattern_free(kv.second->pat);
    for (PatternObj* P : to_free) pattern_free(P);
    to_free.clear();
}

void ServerObj::analysis_loop() {
    cudaSetDevice(device);
    while (true) {
        PatternEntry* pe = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_analysis.wait(lk, [this] { return stopping || !analysis_q.empty(); });
            if (analysis_q.empty()) return;
            pe = analysis_q.front();
            analysis_q.pop_front();
        }
        PatternObj* P = nullptr;
        const int rc = pattern_build(pe->n, pe->Ap.data(), pe->Ai.data(), pe->Ax.data(), nullptr, &P);
        {
            std::lock_guard<std::mutex> lk(mu);
            if (rc == LUSP_OK && P->bytes > pattern_budget) {
                // Admission: a pattern larger than the cache's whole share
                // of the HBM budget is refused (its requests complete with
                // LUSP_EALLOC); its device copy leaves when nothing runs.
                to_free.push_back(P);
                pe->state = PAT_FAILED;
                pe->fail_rc = LUSP_EALLOC;
                stats.refused++;
            } else if (rc == LUSP_OK) {
                pe->pat = P;
                pe->state = PAT_READY;
                pattern_bytes += P->bytes;
                stats.patterns_resident++;
                evict_if_needed();
            } else {
                pe->state = PAT_FAILED;
                pe->fail_rc = rc;
            }
            pe->Ax.clear();
            pe->Ax.shrink_to_fit();
        }
        cv_sched.notify_all();
        cv_done.notify_all();
    }
}

// A request is done with pe: one analysed for that request's own values
// leaves the device at once.  Called with mu held.
void ServerObj::release(PatternEntry* pe) {
    pe->users--;
    if (!pe->own || pe->users > 0 || pe->state == PAT_PENDING) return;
    auto range = patterns.equal_range(pe->key);
    for (auto it = range.first; it != range.second; ++it) {
        if (it->second.get() != pe) continue;
        if (pe->pat) {
            pattern_bytes -= pe->pat->bytes;
            to_free.push_back(pe->pat);
            stats.patterns_resident--;
        }
        patterns.erase(it);
        return;
    }
}

// Least recently used patterns with no request referencing them leave the
// device while the cache exceeds its share of the HBM budget.
void ServerObj::evict_if_needed() {
    while (pattern_bytes > pattern_budget) {
        PatternEntry* victim = nullptr;
        decltype(patterns)::iterator vit;
        for (auto it = patterns.begin(); it != patterns.end(); ++it) {
            PatternEntry* pe = it->second.get();
            if (pe->state != PAT_READY || pe->users > 0) continue;
            if (!victim || pe->last_use < victim->last_use) {
                victim = pe;
                vit = it;
            }
        }
        if (!victim) return;
        pattern_bytes -= victim->pat->bytes;
        to_free.push_back(victim->pat);
        patterns.erase(vit);
        stats.evictions++;
        stats.patterns_resident--;
    }
}

// Pack the oldest ready requests of one mode into this stream's arena and
// launch them.  Called with mu held.
bool ServerObj::try_launch(Flight& f) {
    // Requests whose pattern failed analysis complete at once.
    for (auto it = queue.begin(); it != queue.end();) {
        Request* r = *it;
        if (r->pe->state == PAT_FAILED) {
            r->res.rc = r->pe->fail_rc;
            r->res.status = r->pe->fail_rc == LUSP_EALLOC ? LUSP_ST_CAPACITY : LUSP_ST_SINGULAR;
            r->t_done = Clock::now();
            r->res.latency_ms = ms_since(r->t_submit, r->t_done);
            r->done = true;
            release(r->pe);
            stats.completed++;
            it = queue.erase(it);
            cv_done.notify_all();
        } else {
            ++it;
        }
    }
    // The oldest ready request sets the launch's mode and size class; large
    // systems may hold all but one stream, so launches of small and medium
    // systems never queue behind them.
    int nlarge = 0;
    for (const Flight& g : flights) nlarge += g.busy && g.cls == 2;
    const bool allow_large = nlarge < std::max(1, (int)flights.size() - 1);
    int mode = -1, cls = -1;
    for (Request* r : queue)
        if (r->pe->state == PAT_READY && (allow_large || size_class(r->n) != 2)) {
            mode = r->mode;
            cls = size_class(r->n);
            break;
        }
    if (mode < 0) return false;
    lusp_batch_opts o = opts.solver;
    o.prec = fp64_mode(mode) ? LUSP_FP64 : LUSP_MIXED;
    o.inner_prec = mode == MODE_MIXED_INNER64 ? 1 : (opts.solver.inner_prec == 2 ? 2 : 0);
    const size_t vs = o.prec == LUSP_FP64 ? 8 : 4;
    // Choose requests (FIFO among ready ones of this mode) that fit.
    std::vector<Request*> pick;
    std::vector<PatternObj*> pats;
    size_t up_bytes = 0, down_bytes = 0, priv = 0;
    const int maxb = std::max(1, cls == 2 ? std::min(opts.max_batch, kLargeBatch) : opts.max_batch);
    for (Request* r : queue) {
        if ((int)pick.size() >= maxb) break;
        if (r->pe->state != PAT_READY || r->mode != mode || size_class(r->n) != cls) continue;
        const StaticPattern& S = r->pe->pat->S;
        const size_t up = (r->vals.size() + r->rhs.size()) * 8;
        const size_t down = (size_t)S.n * 8 + sizeof(SysStats);
        const size_t pv = system_private_bytes(S, vs, o.krylov);
        const size_t io = al((up_bytes + up) + (size_t)(S.n + 64) * 8);
        const bool fits = up_bytes + up + down_bytes + down + 4096 <= f.stage_bytes &&
                          priv + pv + io + al(sizeof(SysDev) * (pick.size() + 1)) +
                                  al(sizeof(SysStats) * (pick.size() + 1)) + (64u << 20) <=
                              f.arena_bytes;
        if (!fits && pick.empty()) {
            // Larger than a whole stream arena or staging area: refuse it.
            r->res.rc = LUSP_EALLOC;
            r->res.status = LUSP_ST_CAPACITY;
            r->t_done = Clock::now();
            r->res.latency_ms = ms_since(r->t_submit, r->t_done);
            r->done = true;
            release(r->pe);
            stats.completed++;
            queue.erase(std::find(queue.begin(), queue.end(), r));
            cv_done.notify_all();
            return true;
        }
        if (!fits) break;
        pick.push_back(r);
        pats.push_back(r->pe->pat);
        up_bytes += up;
        down_bytes += down;
        priv += pv;
    }
    if (pick.empty()) return false;
    // Launch shapes and arena layout; drop requests from the back of the
    // pick until everything (including the refactor spill area) fits.
    SmemPlan plan;
    LaunchArgs la;
    LadderPlan lp;
    int grid = 0;
    size_t nval = 0, nvec = 0, spill = 0, syncb = 0;
    const lusp_batch_opts o_req = o;
    while (true) {
        const int nsp = (int)pick.size();
        o = o_req;
        resolve_solve_shape(o, nsp);
        nval = nvec = 0;
        size_t privs = 0;
        int cm = 0;
        for (Request* r : pick) {
            nval += r->vals.size();
            nvec += r->rhs.size();
            privs += system_private_bytes(r->pe->pat->S, vs, o.krylov);
            cm = std::max(cm, r->pe->pat->S.max_col);
        }
        if (plan_for(pats, o, plan) != LUSP_OK) {
            o.solve_sweep = 0;
            plan_for(pats, o, plan);
        }
        int occ = 0;
        if (kernel_occupancy(o.prec, o.inner_prec, plan.bytes, o.block_threads, &occ) != LUSP_OK || occ < 1)
            return false;
        grid = std::min(nsp, occ * sm_count());
        if (refactor_setup(pats, o, nsp, la) != LUSP_OK) return false;
        syncb = la.rspread.group > 0 ? al((size_t)nsp * la.rspread.stride * sizeof(unsigned)) : 0;
        spill = spill_bytes(la.rgrid, la.rblock, cm, la.rplan);
        // Device-side escalation of the mixed path: a few ladder slots with
        // room for the largest systems of the launch.
        la.rungs = 0;
        lp = LadderPlan{};
        const int rungs = fp64_mode(mode) ? 0 : opts.escalate == 1 ? 1 : opts.escalate == 2 ? 3 : 0;
        if (rungs) {
            lusp_batch_opts lo = o;
            lo.ladder = rungs;
            const int cap = std::min(nsp, std::max(4, (nsp + 7) / 8));
            std::vector<size_t> sz;
            for (Request* r : pick) sz.push_back(system_private_bytes(r->pe->pat->S, 8, o.krylov));
            std::sort(sz.begin(), sz.end(), std::greater<size_t>());
            size_t pool = 0;
            for (int i = 0; i < cap; i++) pool += sz[i];
            if (ladder_setup(pats, lo, cap, la, lp, pool) != LUSP_OK) return false;
        }
        const size_t total = al(nval * 8) + 2 * al(nvec * 8) + privs + spill + al(sizeof(SysStats) * nsp) +
                             al(sizeof(SysDev) * nsp) + 256 + lp.bytes + syncb;
        if (total <= f.arena_bytes) break;
        if (nsp == 1) {
            Request* r = pick[0];
            r->res.rc = LUSP_EALLOC;
            r->res.status = LUSP_ST_CAPACITY;
            r->t_done = Clock::now();
            r->res.latency_ms = ms_since(r->t_submit, r->t_done);
            r->done = true;
            release(r->pe);
            stats.completed++;
            queue.erase(std::find(queue.begin(), queue.end(), r));
            cv_done.notify_all();
            return true;
        }
        pick.pop_back();
        pats.pop_back();
    }
    const int ns = (int)pick.size();
    // Arena layout: values | rhs | x | per-system private | spill | stats | descriptors | queue.
    char* a = f.arena;
    double* d_vals = (double*)a;
    double* d_rhs = (double*)(a + al(nval * 8));
    double* d_x = (double*)(a + al(nval * 8) + al(nvec * 8));
    char* p = a + al(nval * 8) + 2 * al(nvec * 8);
    std::vector<SysDev> hs(ns);
    size_t ov = 0, ob = 0;
    f.x_off.assign(ns, 0);
    for (int i = 0; i < ns; i++) {
        Request* r = pick[i];
        SysDev& D = hs[i];
        D.pat = r->pe->pat->d_desc;
        D.a_val = d_vals + ov;
        D.b = d_rhs + ob;
        D.x = d_x + ob;
        f.x_off[i] = ob;
        p = carve_system(D, p, r->pe->pat->S, vs, o.krylov);
        ov += r->vals.size();
        ob += r->rhs.size();
    }
    double* d_spill = spill ? (double*)p : nullptr;
    p += spill;
    SysStats* d_stats = (SysStats*)p;
    p += al(sizeof(SysStats) * ns);
    SysDev* d_sys = (SysDev*)p;
    p += al(sizeof(SysDev) * ns);
    int* d_queue = (int*)p;
    p += 256;
    char* d_ladder = p;
    p += lp.bytes;
    // Spread mode: the systems' sync areas (zeroed by the launch).
    if (syncb) la.rspread.sync = (unsigned*)p;
    p += syncb;
    if ((size_t)(p - a) > f.arena_bytes) return false;
    ladder_bind(la, lp, d_ladder, d_queue);
    for (int i = 0; i < ns; i++) {
        hs[i].scratch = d_spill;
        hs[i].stats = d_stats + i;
    }
    // Stage the inputs in pinned memory and move them in one copy.
    char* up = f.stage;
    size_t o2 = 0;
    for (Request* r : pick) {
        std::memcpy(up + o2, r->vals.data(), r->vals.size() * 8);
        o2 += r->vals.size() * 8;
    }
    const size_t rhs_at = o2;
    for (Request* r : pick) {
        std::memcpy(up + o2, r->rhs.data(), r->rhs.size() * 8);
        o2 += r->rhs.size() * 8;
    }
    f.down_x = al(o2);
    f.down_stats = al(f.down_x + nvec * 8);
    const auto now = Clock::now();
    cudaError_t e = cudaEventRecord(f.ev0, f.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_vals, up, nval * 8, cudaMemcpyHostToDevice, f.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rhs, up + rhs_at, nvec * 8, cudaMemcpyHostToDevice, f.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_sys, hs.data(), sizeof(SysDev) * ns, cudaMemcpyHostToDevice, f.st);
    if (e != cudaSuccess) return false;
    la.d_sys = d_sys;
    la.nsys = ns;
    la.d_queue = d_queue;
    la.plan = plan;
    fill_params(la.prm, o);
    la.prec = o.prec;
    la.inner = o.inner_prec;
    la.ir64 = mode == MODE_FP64_IR ? 1 : 0;
    la.what = LUSP_RUN_BOTH;
    la.block = o.block_threads;
    la.grid = grid;
    if (launch_systems(la, f.st) != LUSP_OK) return false;
    e = cudaMemcpyAsync(f.stage + f.down_x, d_x, nvec * 8, cudaMemcpyDeviceToHost, f.st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(f.stage + f.down_stats, d_stats, sizeof(SysStats) * ns, cudaMemcpyDeviceToHost, f.st);
    if (e == cudaSuccess) e = cudaEventRecord(f.ev1, f.st);
    if (e != cudaSuccess) return false;
    // Hand the requests to the flight.
    f.reqs = pick;
    f.busy = true;
    f.cls = cls;
    for (Request* r : pick) {
        r->t_launch = now;
        r->res.batch_size = ns;
    }
    queue.erase(std::remove_if(queue.begin(), queue.end(),
                               [&pick](Request* r) { return std::find(pick.begin(), pick.end(), r) != pick.end(); }),
                queue.end());
    stats.launches++;
    stats.max_batch_seen = std::max<long long>(stats.max_batch_seen, ns);
    return true;
}

// A flight finished: publish results, re-queue systems that need the fp64
// path.  Called with mu held.
void ServerObj::complete(Flight& f) {
    float dev_ms = 0.f;
    cudaEventElapsedTime(&dev_ms, f.ev0, f.ev1);
    const SysStats* st = (const SysStats*)(f.stage + f.down_stats);
    const double* xs = (const double*)(f.stage + f.down_x);
    const auto now = Clock::now();
    const int fail = LUSP_ST_SINGULAR | LUSP_ST_PIVOT_WEAK | LUSP_ST_STAGNATED | LUSP_ST_NOT_CONVERGED |
                     LUSP_ST_NONFINITE | LUSP_ST_WAIT_TIMEOUT | LUSP_ST_CAPACITY;
    for (size_t i = 0; i < f.reqs.size(); i++) {
        Request* r = f.reqs[i];
        const SysStats& s = st[i];
        const bool failed = (s.status & fail) != 0 ||
                            (!fp64_mode(r->mode) && s.nres > 0 && !(s.res[s.nres - 1] <= opts.solver.rtol));
        // The last step of the ladder: an fp64 solve that still fails with
        // the frozen pivots (chosen for the pattern's first values) is
        // analysed again with this request's own values (fresh partial
        // pivoting) and solved once more with an fp64 factor and GMRES-IR.
        const int hard = LUSP_ST_SINGULAR | LUSP_ST_STAGNATED | LUSP_ST_NOT_CONVERGED | LUSP_ST_NONFINITE;
        const bool fp64_failed = (s.rung > 0 || r->mode == MODE_FP64_IR) &&
                                 ((s.status & hard) != 0 || !(s.nres > 0 && s.res[s.nres - 1] <= opts.solver.rtol));
        // The outcome of a request's mixed attempt updates its pattern's
        // escalation memory (r->pe is still the shared pattern here: only an
        // fp64 attempt re-pivots).
        if (!r->learned && !fp64_mode(r->mode) && opts.escalate) {
            r->learned = true;
            PatternEntry* pe = r->pe;
            if (s.rung > 0 || failed) {
                if (++pe->esc_run >= 2 && !pe->promoted) {
                    pe->promoted = true;
                    pe->since_trial = 0;
                    stats.promoted++;
                }
            } else {
                pe->esc_run = 0;
                if (r->trial && pe->promoted) pe->promoted = false;
            }
        }
        if (fp64_failed && !r->repivoted && opts.escalate) {
            auto npe = std::make_unique<PatternEntry>();
            npe->key = r->pe->key;
            npe->n = r->n;
            npe->Ap = r->pe->Ap;
            npe->Ai = r->pe->Ai;
            npe->Ax = r->vals;
            npe->own = true;
            npe->users = 1;
            npe->last_use = ++clock;
            PatternEntry* pe2 = npe.get();
            patterns.emplace(npe->key, std::move(npe));
            analysis_q.push_back(pe2);
            cv_analysis.notify_one();
            release(r->pe);
            r->pe = pe2;
            r->mode = MODE_FP64_IR;
            r->repivoted = true;
            if (!r->escalated) stats.escalated++;
            r->escalated = true;
            queue.push_front(r);
            continue;
        }
        if (s.rung > 0) {
            // Escalated on the device in the same launch: final.
            r->escalated = true;
            stats.escalated++;
        } else if (failed && !fp64_mode(r->mode) && opts.escalate) {
            // Not taken by a ladder (none, or no slot left): once more with
            // an fp64 factor and GMRES-IR in a launch of its own.
            r->mode = MODE_FP64_IR;
            r->escalated = true;
            queue.push_front(r);
            stats.escalated++;
            continue;
        }
        r->x.assign(xs + f.x_off[i], xs + f.x_off[i] + r->n);
        r->t_done = now;
        r->res.rc = LUSP_OK;
        r->res.status = s.status | (r->escalated ? LUSP_ST_ESCALATED : 0);
        r->res.latency_ms = ms_since(r->t_submit, now);
        r->res.queue_ms = ms_since(r->t_submit, r->t_launch);
        r->res.device_ms = dev_ms;
        r->res.residual = s.nres > 0 ? s.res[s.nres - 1] : -1.0;
        r->res.inner_iters = s.inner_iters;
        r->res.outer_iters = s.outer_iters;
        r->res.cache_hit = r->cache_hit ? 1 : 0;
        r->res.escalated = r->escalated ? 1 : 0;
        r->res.pattern_hash = r->pe->key;
        r->pe->last_use = ++clock;
        release(r->pe);
        r->pe = nullptr;
        r->done = true;
        stats.completed++;
    }
    f.reqs.clear();
    f.busy = false;
    evict_if_needed();
}

void ServerObj::sched_loop() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        bool progress = false;
        for (auto& f : flights) {
            if (f.busy && cudaEventQuery(f.ev1) == cudaSuccess) {
                complete(f);
                progress = true;
            }
        }
        for (auto& f : flights) {
            if (!f.busy && !queue.empty() && try_launch(f)) progress = true;
        }
        if (progress) cv_done.notify_all();
        bool busy = false;
        for (auto& f : flights) busy |= f.busy;
        if (!busy && !to_free.empty()) {
            // Nothing in flight: a free here waits for no kernel.
            for (PatternObj* P : to_free) pattern_free(P);
            to_free.clear();
        }
        if (stopping && !busy && queue.empty()) return;
        if (!progress) {
            // Poll completions every 20 us while work is in flight; sleep
            // until a submission otherwise.
            if (busy) cv_sched.wait_for(lk, std::chrono::microseconds(20));
            else cv_sched.wait_for(lk, std::chrono::milliseconds(5));
        }
    }
}

}  // namespace lusp

using lusp::ServerObj;

static ServerObj* SO(lusp_server* s) { return reinterpret_cast<ServerObj*>(s); }

extern "C" {

void lusp_server_opts_default(lusp_server_opts* o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    lusp_batch_opts_default(&o->solver);
    o->max_batch = 128;
    o->streams = 3;
    o->hbm_budget_gb = 150.0;
    o->arena_gb = 2.0;
    o->staging_mb = 256.0;
    o->escalate = 1;
    o->analysis_threads = 4;
}

int lusp_server_create(const lusp_server_opts* o, lusp_server** out) {
    if (!out) return LUSP_EARG;
    *out = nullptr;
    lusp_server_opts d;
    if (o) d = *o; else lusp_server_opts_default(&d);
    int rc = lusp::check_opts(&d.solver);
    if (rc != LUSP_OK) return rc;
    if (d.arena_gb <= 0 || d.staging_mb <= 0 || d.max_batch <= 0) return LUSP_EARG;
    ServerObj* S = nullptr;
    try {
        S = new ServerObj();
    } catch (const std::bad_alloc&) {
        return LUSP_EALLOC;
    }
    S->opts = d;
    rc = S->init();
    if (rc != LUSP_OK) {
        S->shutdown();
        delete S;
        return rc;
    }
    *out = reinterpret_cast<lusp_server*>(S);
    return LUSP_OK;
}

void lusp_server_destroy(lusp_server* s) {
    ServerObj* S = SO(s);
    if (!S) return;
    S->shutdown();
    delete S;
}

long long lusp_serve_submit(lusp_server* s, int n, const int* Ap, const int* Ai, const double* Ax,
                            const double* b) {
    ServerObj* S = SO(s);
    if (!S || n <= 0 || !Ap || !Ai || !Ax || !b) return -LUSP_EARG;
    const int nnz = Ap[n];
    if (Ap[0] != 0 || nnz < 0) return -LUSP_EARG;
    try {
        auto r = std::make_unique<lusp::Request>();
        r->n = n;
        r->vals.assign(Ax, Ax + nnz);
        r->rhs.assign(b, b + n);
        r->t_submit = lusp::Clock::now();
        r->mode = S->opts.solver.prec == LUSP_FP64 ? lusp::MODE_FP64
                                                    : (S->opts.solver.inner_prec == 1 ? lusp::MODE_MIXED_INNER64
                                                                                       : lusp::MODE_MIXED);
        const uint64_t key = lusp::structure_hash(n, Ap, Ai);
        std::lock_guard<std::mutex> lk(S->mu);
        lusp::PatternEntry* pe = nullptr;
        auto range = S->patterns.equal_range(key);
        for (auto it = range.first; it != range.second; ++it) {
            lusp::PatternEntry* c = it->second.get();
            if (!c->own && c->n == n && (int)c->Ai.size() == nnz && std::equal(c->Ap.begin(), c->Ap.end(), Ap) &&
                std::equal(c->Ai.begin(), c->Ai.end(), Ai)) {
                pe = c;
                break;
            }
        }
        if (pe) {
            r->cache_hit = true;
            S->stats.cache_hits++;
            // A pattern whose mixed requests keep escalating starts on the
            // fp64 factor + GMRES-IR path, with a mixed trial now and then.
            if (pe->promoted && !lusp::fp64_mode(r->mode)) {
                if (++pe->since_trial >= lusp::kTrialEvery) {
                    pe->since_trial = 0;
                    r->trial = true;
                } else {
                    r->mode = lusp::MODE_FP64_IR;
                    S->stats.fp64_starts++;
                }
            }
        } else {
            auto npe = std::make_unique<lusp::PatternEntry>();
            npe->key = key;
            npe->n = n;
            npe->Ap.assign(Ap, Ap + n + 1);
            npe->Ai.assign(Ai, Ai + nnz);
            npe->Ax.assign(Ax, Ax + nnz);
            pe = npe.get();
            S->patterns.emplace(key, std::move(npe));
            S->analysis_q.push_back(pe);
            S->stats.cache_misses++;
            S->cv_analysis.notify_one();
        }
        pe->users++;
        pe->last_use = ++S->clock;
        r->pe = pe;
        const long long id = S->next_id++;
        r->id = id;
        S->queue.push_back(r.get());
        S->reqs.emplace(id, std::move(r));
        S->stats.submitted++;
        S->cv_sched.notify_one();
        return id;
    } catch (const std::bad_alloc&) {
        return -LUSP_EALLOC;
    }
}

int lusp_serve_poll(lusp_server* s, long long id, double* x, lusp_serve_result* res, int wait_ms) {
    ServerObj* S = SO(s);
    if (!S) return LUSP_EARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return LUSP_EARG;
    lusp::Request* r = it->second.get();
    if (!r->done) {
        if (wait_ms == 0) return LUSP_EBUSY;
        auto ready = [r] { return r->done; };
        if (wait_ms < 0) S->cv_done.wait(lk, ready);
        else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready)) return LUSP_EBUSY;
    }
    if (x && !r->x.empty()) std::memcpy(x, r->x.data(), sizeof(double) * r->n);
    if (res) *res = r->res;
    S->reqs.erase(it);
    return LUSP_OK;
}

int lusp_server_get_stats(lusp_server* s, lusp_server_stats* st) {
    ServerObj* S = SO(s);
    if (!S || !st) return LUSP_EARG;
    std::lock_guard<std::mutex> lk(S->mu);
    *st = S->stats;
    st->pattern_gb = S->pattern_bytes / 1e9;
    return LUSP_OK;
}

}  // extern "C"
