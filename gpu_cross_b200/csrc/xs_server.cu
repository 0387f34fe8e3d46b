// Request server: continuous batching of cross-section requests over line
// lists kept resident in HBM.  No counterpart in the reference (which runs
// one .inp job per process); it serves the same arithmetic per request.
//
// A request names a resident molecule, T, Q(T), P, a profile and a uniform
// grid.  Its grid is planned into chunks of whole 256-point tiles, each with
// the slice of lines that can reach it and bounded work, so that no chunk
// holds the GPU for long.  A scheduler thread
//   * admits queued requests (FIFO) while their device and pinned-host
//     memory fit the budgets, giving each a lane (stream + engine) and
//     filling its grid and zeroing its output on that stream;
//   * issues chunks, at most as many in flight as there are lanes: each
//     time the request with the least remaining work over all lanes (its
//     lane having room), so small requests that arrive while a large one
//     runs are interleaved between its chunks and finish early, and a large
//     one runs at the GPU's full rate when nothing smaller waits;
//   * after a request's last chunk, copies its result to pinned host memory
//     and, when that copy's event completes, releases its memory and wakes
//     the waiter.
// Work from different lanes may overlap on the device.  A request's chunks
// depend only on the request itself, so its result is bit-identical whether
// it runs alone or in a mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "xs_engine.h"
#include "xsec_b200.h"

namespace xs {
cudaError_t partition_on_stream(const double* d_e, const int* d_g, long n, const double* d_beta,
                                int n_temps, double* d_q, double* work, cudaStream_t stream);
size_t partition_work_doubles(int n_temps);
double partition_beta(double temperature);
}  // namespace xs

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

int sfail(int code, const std::string& msg) { return xs::set_error(code, msg.c_str()); }

// f[i] = f0 + i*df with one rounding per operation (no fused multiply-add),
// the grid BaseProfile builds (BaseProfile.cpp:17-21).
__global__ void k_fill_grid(double* f, double f0, double df, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = __dadd_rn(f0, __dmul_rn(double(i), df));
}

constexpr int kTile = 256;  // chunk granularity: a multiple of every tile width
// Molecules per server.  The scheduler reads the molecule table without the
// lock; reserving it up front keeps its elements in place while
// xs_server_add_molecule appends.
constexpr size_t kMaxMolecules = 64;

// ---------------------------------------------------------------------------
// Chunk planning (host only).
//
// Line-evals of a 256-point tile [a, b] (a = f_s - df/2, b = f_e-1 + df/2)
// are estimated as the summed overlap of the windows [nu - cut, nu + cut]
// with [a, b], divided by df.  On each interval between the four breakpoints
// a -/+ cut, b -/+ cut the overlap is linear in nu, so prefix sums of nu
// give the sum from four lower-bound positions; the sum is additive over
// tiles.  The breakpoints only move up from tile to tile, so each position
// is found by a galloping search from the previous tile's.
struct LineIndex {
    const double* nu = nullptr;   // ascending
    const double* cum = nullptr;  // cum[k] = sum of nu[0..k)
    size_t n = 0;

    size_t lower(double v) const { return size_t(std::lower_bound(nu, nu + n, v) - nu); }
    size_t upper(double v) const { return size_t(std::upper_bound(nu, nu + n, v) - nu); }
};

// First index with nu[i] >= v (strict = false) or nu[i] > v (strict = true),
// for nondecreasing v.
struct Cursor {
    size_t pos = 0;
    size_t seek(const LineIndex& L, double v, bool strict) {
        auto before = [&](size_t i) { return strict ? !(L.nu[i] > v) : L.nu[i] < v; };
        if (pos >= L.n || !before(pos)) return pos;
        size_t lo = pos, step = 1, hi;
        for (;;) {  // before(lo) holds
            hi = lo + step;
            if (hi >= L.n) {
                hi = L.n;
                break;
            }
            if (!before(hi)) break;
            lo = hi;
            step *= 2;
        }
        const double* first = L.nu + lo + 1;
        const double* last = L.nu + hi;
        pos = size_t((strict ? std::upper_bound(first, last, v) : std::lower_bound(first, last, v)) - L.nu);
        return pos;
    }
};

double overlap_sum(const LineIndex& L, const size_t idx[4], const double p[4], double a, double b,
                   double cut) {
    double sum = 0.0;
    for (int k = 0; k < 3; ++k) {
        if (!(p[k + 1] > p[k])) continue;
        const size_t i0 = idx[k], i1 = idx[k + 1];
        if (i1 <= i0) continue;
        const double mid = 0.5 * (p[k] + p[k + 1]);
        const bool min_nu = mid + cut < b;  // min(nu + cut, b) is nu + cut
        const bool max_nu = mid - cut > a;  // max(nu - cut, a) is nu - cut
        const double slope = (min_nu ? 1.0 : 0.0) - (max_nu ? 1.0 : 0.0);
        const double icpt = (min_nu ? cut : b) - (max_nu ? -cut : a);
        const double v = slope * (L.cum[i1] - L.cum[i0]) + icpt * double(i1 - i0);
        if (v > 0.0) sum += v;
    }
    return sum;
}

struct ChunkPlan {
    int start, points;
    size_t l0, l1;  // line slice
    double pairs;   // estimated line-evals inside the window (what is reported)
    double cost;    // estimated work: line-evals inside the cost window
};

// Greedy over tiles: a chunk takes tiles while its estimated work stays
// within max_pairs and its line slice within max_lines (at least one tile).
// The work is counted over [nu - cost_cut, nu + cost_cut]: the window for
// Voigt, the span where Doppler pairs are not skipped as exact zeros.
void plan_chunks(const LineIndex& L, double f0, double df, int npoints, double cut,
                 double cost_cut, double max_pairs, size_t max_lines, std::vector<ChunkPlan>& out) {
    out.clear();
    const double margin = 2.0 * df;
    auto freq = [&](long i) { return f0 + double(i) * df; };
    Cursor bp[4], bq[4], c_lo, c_hi;
    const int ntiles = (npoints + kTile - 1) / kTile;
    ChunkPlan cur{0, 0, 0, 0, 0.0, 0.0};
    auto tile_sum = [&](Cursor* cs, double a, double b, double h) {
        // breakpoints in ascending order; a + h and b - h swap when the tile
        // is wider than the window
        double p[4] = {a - h, std::min(a + h, b - h), std::max(a + h, b - h), b + h};
        size_t idx[4];
        for (int k = 0; k < 4; ++k) idx[k] = cs[k].seek(L, p[k], false);
        return overlap_sum(L, idx, p, a, b, h) / df;
    };
    for (int t = 0; t < ntiles; ++t) {
        const int s = t * kTile, e = std::min(npoints, s + kTile);
        const double a = freq(s) - 0.5 * df, b = freq(e - 1) + 0.5 * df;
        const double tp = tile_sum(bp, a, b, cut);
        const double tc = cost_cut < cut ? tile_sum(bq, a, b, cost_cut) : tp;
        const size_t l1 = c_hi.seek(L, freq(e - 1) + cut + margin, true);
        if (cur.points > 0 && (cur.cost + tc > max_pairs || l1 - cur.l0 > max_lines)) {
            out.push_back(cur);
            cur = ChunkPlan{s, 0, 0, 0, 0.0, 0.0};
        }
        if (cur.points == 0) {
            cur.start = s;
            cur.l0 = c_lo.seek(L, freq(s) - cut - margin, false);
        }
        cur.points = e - cur.start;
        cur.l1 = l1;
        cur.pairs += tp;
        cur.cost += tc;
    }
    out.push_back(cur);
}

// ---------------------------------------------------------------------------
// First-fit allocator over one pinned host arena.
class Arena {
public:
    bool init(size_t bytes) {
        if (cudaHostAlloc(&base_, bytes, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            base_ = nullptr;
            return false;
        }
        size_ = bytes;
        free_[0] = bytes;
        return true;
    }
    void release() {
        if (base_) cudaFreeHost(base_);
        base_ = nullptr;
        free_.clear();
    }
    // Returns the offset, or SIZE_MAX when nothing fits.
    size_t alloc(size_t bytes) {
        bytes = (bytes + 255) & ~size_t(255);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                const size_t off = it->first, left = it->second - bytes;
                free_.erase(it);
                if (left) free_[off + bytes] = left;
                used_ += bytes;
                return off;
            }
        }
        return SIZE_MAX;
    }
    void free(size_t off, size_t bytes) {
        bytes = (bytes + 255) & ~size_t(255);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
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
    double* at(size_t off) { return reinterpret_cast<double*>(static_cast<char*>(base_) + off); }
    size_t size() const { return size_; }

private:
    void* base_ = nullptr;
    size_t size_ = 0, used_ = 0;
    std::map<size_t, size_t> free_;
};

struct Molecule {
    double *nu = nullptr, *e = nullptr, *a = nullptr, *g = nullptr, *nx = nullptr;
    int* gns = nullptr;
    size_t n = 0;
    double mass = 0.0, ref_temp = 296.0;
    std::vector<double> h_nu, h_cum;
    size_t bytes = 0;
    // optional state list (xs_server_add_states) for Q(T), cached per T
    double* d_se = nullptr;
    int* d_sg = nullptr;
    size_t ns = 0;
    std::map<double, double> qcache;
    LineIndex index() const {
        LineIndex L;
        L.nu = h_nu.data();
        L.cum = h_cum.data();
        L.n = n;
        return L;
    }
};

// Per-temperature intensity cache of one molecule, profile, T and Q(T):
// S(T) and, for Voigt, (T_ref/T)^n of every line, as step one computes them.
// `covered`: line ranges stored by completed chunks (sorted, disjoint).
struct TCache {
    int mol = -1, profile = 0;
    double T = 0.0, Q = 0.0;
    double* s = nullptr;
    double* pw = nullptr;
    size_t bytes = 0;
    std::vector<std::pair<size_t, size_t>> covered;
    int refs = 0;                 // admitted requests that use it
    unsigned long long used = 0;  // last use (least recently used goes first)
    bool covers(size_t l0, size_t l1) const {
        for (const auto& c : covered)
            if (c.first <= l0 && l1 <= c.second) return true;
        return false;
    }
    void add(size_t l0, size_t l1) {
        covered.emplace_back(l0, l1);
        std::sort(covered.begin(), covered.end());
        std::vector<std::pair<size_t, size_t>> m;
        for (const auto& c : covered) {
            if (!m.empty() && c.first <= m.back().second)
                m.back().second = std::max(m.back().second, c.second);
            else
                m.push_back(c);
        }
        covered.swap(m);
    }
};

// XS_POLICY_DEADLINE: estimated line-evals the device runs per millisecond
// (a request's deadline is its submission time plus its remaining work at
// this rate).
constexpr double kDeadlineRate = 2.0e9;

struct Request {
    unsigned long long id = 0;
    xs_request q{};
    xs_options opt{};
    xs_condition cond{};
    std::vector<ChunkPlan> chunks;
    size_t next = 0;
    int lane = -1;
    double remaining = 0.0, pairs = 0.0;
    size_t lines = 0;
    double* d_freq = nullptr;
    double* d_out = nullptr;
    size_t dev_bytes = 0, host_off = SIZE_MAX, host_bytes = 0;
    Clock::time_point t_submit, t_admit, t_done;
    unsigned long long last_issue = 0;  // round robin: issue order of its last chunk
    int tc = -1;                        // per-temperature cache in use (index)
    int tc_chunks = 0;                  // chunks that read it
    int status = XS_OK;
    std::string error;
    bool done = false;
};

struct Flight {
    Request* r;
    cudaEvent_t ev;
    bool last;
    int tc_wrote;        // cache the chunk stored into (-1: none) ...
    size_t l0, l1;       // ... for these lines
};

struct Lane {
    xs_engine* eng = nullptr;
    cudaStream_t st = nullptr;
    std::deque<Flight> flight;
    double load = 0.0;  // remaining line-evals of the requests assigned here
};

}  // namespace

struct xs_server {
    int device = 0;
    xs_server_config cfg{};
    size_t resident = 0;        // molecules + lane scratch
    size_t dev_requests = 0;    // grids + outputs of admitted requests
    std::vector<Molecule> mols;
    std::vector<Lane> lanes;
    unsigned long long issue_seq = 0;  // chunks issued (round robin order)
    // per-temperature caches (scheduler-owned); keys seen once are remembered
    // so that a cache is made on a key's second request
    std::vector<TCache> tcache;
    size_t tc_used = 0;
    unsigned long long tc_clock = 0;
    std::deque<std::tuple<int, int, double, double>> tc_seen;
    Arena arena;
    std::vector<cudaEvent_t> ev_pool;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> incoming;             // submitted, not yet seen by the scheduler
    std::map<unsigned long long, Request*> all; // not yet collected by xs_server_wait
    unsigned long long next_id = 1;
    std::string fatal;

    std::deque<Request*> queue;   // scheduler-owned: waiting for admission
    std::vector<Request*> active; // scheduler-owned: admitted, not finished
    std::thread worker;
    std::atomic<bool> stop{false};
    std::atomic<int> n_queued{0}, n_active{0};

    // partition functions of molecules with states: one at a time
    std::mutex qmu;
    cudaStream_t aux = nullptr;
    double* d_pwork = nullptr;  // beta, Q and the block sums of one temperature
};

namespace {

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DevGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

size_t request_device_bytes(const xs_request& q) {
    const size_t b = sizeof(double) * size_t(q.npoints);
    return 2 * ((b + 511) & ~size_t(511));
}

cudaEvent_t take_event(xs_server* s) {
    if (!s->ev_pool.empty()) {
        cudaEvent_t e = s->ev_pool.back();
        s->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}

// Frees a per-temperature cache that no request holds (cudaFree waits for
// the device; caches are made and dropped rarely: on a key's second request,
// and when room is needed).
void tc_drop(xs_server* s, size_t k) {
    TCache& e = s->tcache[k];
    cudaFree(e.s);
    s->tc_used -= e.bytes;
    e = TCache{};
}

// Drops the least recently used cache that no request holds; false when
// there is none.
bool tc_drop_lru(xs_server* s) {
    int victim = -1;
    for (size_t k = 0; k < s->tcache.size(); ++k) {
        const TCache& e = s->tcache[k];
        if (e.s && e.refs == 0 && (victim < 0 || e.used < s->tcache[size_t(victim)].used)) victim = int(k);
    }
    if (victim < 0) return false;
    tc_drop(s, size_t(victim));
    return true;
}

// The per-temperature cache of an admitted request's key (molecule, profile,
// T, Q): an existing one, or a new one on the key's second request when it
// fits the budgets; -1: none.
int tc_acquire(xs_server* s, Request* r) {
    if (s->cfg.tcache_bytes < 0) return -1;
    const int mol = r->q.molecule, prof = r->q.profile;
    const double T = r->q.temperature, Q = r->cond.partition;
    for (size_t k = 0; k < s->tcache.size(); ++k) {
        TCache& e = s->tcache[k];
        if (e.s && e.mol == mol && e.profile == prof && e.T == T && e.Q == Q) {
            ++e.refs;
            e.used = ++s->tc_clock;
            return int(k);
        }
    }
    const auto key = std::make_tuple(mol, prof, T, Q);
    auto it = std::find(s->tc_seen.begin(), s->tc_seen.end(), key);
    if (it == s->tc_seen.end()) {
        s->tc_seen.push_back(key);
        if (s->tc_seen.size() > 256) s->tc_seen.pop_front();
        return -1;
    }
    s->tc_seen.erase(it);
    const size_t n = s->mols[size_t(mol)].n;
    const size_t bytes = sizeof(double) * n * (prof == XS_VOIGT ? 2 : 1);
    const size_t cap = size_t(s->cfg.tcache_bytes);
    auto fits = [&]() {
        return s->tc_used + bytes <= cap &&
               s->resident + s->dev_requests + s->tc_used + bytes <= s->cfg.device_budget;
    };
    while (!fits())
        if (!tc_drop_lru(s)) return -1;
    double* d = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&d), bytes) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    size_t k = 0;
    while (k < s->tcache.size() && s->tcache[k].s) ++k;
    if (k == s->tcache.size()) s->tcache.emplace_back();
    TCache& e = s->tcache[k];
    e.mol = mol;
    e.profile = prof;
    e.T = T;
    e.Q = Q;
    e.s = d;
    e.pw = prof == XS_VOIGT ? d + n : nullptr;
    e.bytes = bytes;
    e.refs = 1;
    e.used = ++s->tc_clock;
    s->tc_used += bytes;
    return int(k);
}

void finish(xs_server* s, Request* r) {
    Lane& ln = s->lanes[size_t(r->lane)];
    if (r->tc >= 0) --s->tcache[size_t(r->tc)].refs;
    r->tc = -1;
    if (r->d_freq) cudaFreeAsync(r->d_freq, ln.st);
    if (r->d_out) cudaFreeAsync(r->d_out, ln.st);
    r->d_freq = r->d_out = nullptr;
    s->dev_requests -= r->dev_bytes;
    ln.load -= r->remaining;
    r->remaining = 0.0;
    s->active.erase(std::find(s->active.begin(), s->active.end(), r));
    s->n_active = int(s->active.size());
    std::lock_guard<std::mutex> lk(s->mu);
    r->t_done = Clock::now();
    r->done = true;
    s->cv_done.notify_all();
}

// Marks every unfinished request failed (a CUDA error left the context
// unusable) and stops the scheduler.
void fail_all(xs_server* s, const std::string& why) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->fatal = why;
    auto fail_one = [&](Request* r) {
        r->status = XS_ERR_CUDA;
        r->error = why;
        r->t_done = Clock::now();
        r->done = true;
    };
    for (Request* r : s->queue) fail_one(r);
    for (Request* r : s->active) fail_one(r);
    for (Request* r : s->incoming) fail_one(r);
    s->queue.clear();
    s->active.clear();
    s->incoming.clear();
    s->n_active = 0;
    s->n_queued = 0;
    s->cv_done.notify_all();
}

void fail_request(xs_server* s, Request* r, int code, const std::string& why) {
    std::lock_guard<std::mutex> lk(s->mu);
    r->status = code;
    r->error = why;
    r->t_done = Clock::now();
    r->done = true;
    s->cv_done.notify_all();
}

enum class Admit { kAdmitted, kNoRoom, kFailed };

Admit admit(xs_server* s, Request* r) {
    const size_t host = sizeof(double) * size_t(r->q.npoints);
    // requests come before caches: drop caches no request holds for room
    while (s->resident + s->dev_requests + s->tc_used + r->dev_bytes > s->cfg.device_budget)
        if (!tc_drop_lru(s)) return Admit::kNoRoom;
    size_t off;
    {
        std::lock_guard<std::mutex> lk(s->mu);  // the arena is shared with xs_server_wait
        off = s->arena.alloc(host);
    }
    if (off == SIZE_MAX) return Admit::kNoRoom;
    // the lane with the least outstanding work
    size_t li = 0;
    for (size_t k = 1; k < s->lanes.size(); ++k)
        if (s->lanes[k].load < s->lanes[li].load) li = k;
    Lane& ln = s->lanes[li];
    r->lane = int(li);
    r->host_off = off;
    r->host_bytes = host;
    const size_t half = r->dev_bytes / 2;
    cudaError_t err = cudaMallocAsync(reinterpret_cast<void**>(&r->d_freq), half, ln.st);
    if (err == cudaSuccess) err = cudaMallocAsync(reinterpret_cast<void**>(&r->d_out), half, ln.st);
    if (err == cudaSuccess) {
        const int n = r->q.npoints;
        k_fill_grid<<<(n + 255) / 256, 256, 0, ln.st>>>(r->d_freq, r->q.f0, r->q.df, n);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemsetAsync(r->d_out, 0, sizeof(double) * size_t(r->q.npoints), ln.st);
    if (err != cudaSuccess) {
        cudaGetLastError();
        if (r->d_freq) cudaFreeAsync(r->d_freq, ln.st);
        if (r->d_out) cudaFreeAsync(r->d_out, ln.st);
        r->d_freq = r->d_out = nullptr;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->arena.free(off, host);
        }
        r->host_off = SIZE_MAX;
        fail_request(s, r, err == cudaErrorMemoryAllocation ? XS_ERR_NOMEM : XS_ERR_CUDA,
                     std::string("admission: ") + cudaGetErrorString(err));
        return Admit::kFailed;
    }
    s->dev_requests += r->dev_bytes;
    ln.load += r->remaining;
    r->tc = tc_acquire(s, r);
    r->t_admit = Clock::now();
    s->active.push_back(r);
    s->n_active = int(s->active.size());
    return Admit::kAdmitted;
}

// Enqueues the next chunk of r on its lane.  Returns false on a CUDA error
// that leaves the server unusable.
bool issue(xs_server* s, Request* r) {
    Lane& ln = s->lanes[size_t(r->lane)];
    const Molecule& m = s->mols[size_t(r->q.molecule)];
    const ChunkPlan& c = r->chunks[r->next++];
    int wrote = -1;
    if (r->status == XS_OK) {
        xs_lines L;
        L.nu = m.nu + c.l0;
        L.energies = m.e + c.l0;
        L.aif = m.a + c.l0;
        L.gns = m.gns + c.l0;
        L.gamma = m.g + c.l0;
        L.n = m.nx + c.l0;
        L.count = c.l1 - c.l0;
        xs_grid G{r->d_freq, r->q.npoints, c.start, c.points};
        xs::ExecOverride ov;
        ov.no_timing = true;
        if (r->tc >= 0) {
            // step one reads the cached S(T) of lines that completed chunks
            // stored, else computes and stores them
            const TCache& e = s->tcache[size_t(r->tc)];
            ov.tc_s = e.s + c.l0;
            ov.tc_pw = e.pw ? e.pw + c.l0 : nullptr;
            if (e.covers(c.l0, c.l1)) {
                ov.tc_mode = 1;
                ++r->tc_chunks;
            } else {
                ov.tc_mode = 2;
                wrote = r->tc;
            }
        }
        const int rc = xs::engine_execute(ln.eng, &r->opt, &r->cond, 1, &L, &G, r->d_out, 0, &ov);
        if (rc != XS_OK) {
            wrote = -1;  // nothing was stored
            r->status = rc;
            r->error = xs_last_error();
            if (rc == XS_ERR_CUDA) return false;
            r->next = r->chunks.size();  // nothing more to run
        }
    }
    r->remaining -= c.cost;
    ln.load -= c.cost;
    const bool last = r->next >= r->chunks.size();
    if (last && r->status == XS_OK) {
        if (cudaMemcpyAsync(s->arena.at(r->host_off), r->d_out, sizeof(double) * size_t(r->q.npoints),
                            cudaMemcpyDeviceToHost, ln.st) != cudaSuccess)
            return false;
    }
    cudaEvent_t ev = take_event(s);
    if (!ev || cudaEventRecord(ev, ln.st) != cudaSuccess) return false;
    ln.flight.push_back({r, ev, last, wrote, c.l0, c.l1});
    return true;
}

void scheduler(xs_server* s) {
    DevGuard dg(s->device);
    const int depth = s->cfg.depth;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            bool busy = !s->active.empty() || !s->queue.empty();
            if (!busy && s->incoming.empty() && !s->stop)
                s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
            while (!s->incoming.empty()) {
                s->queue.push_back(s->incoming.front());
                s->incoming.pop_front();
            }
            if (s->stop) {
                // shutting down: requests not admitted yet are refused (their
                // memory may be held by results nobody will collect)
                for (Request* r : s->queue) {
                    r->status = XS_ERR_STATE;
                    r->error = "server destroyed before the request was admitted";
                    r->t_done = Clock::now();
                    r->done = true;
                }
                s->queue.clear();
                s->cv_done.notify_all();
            }
            s->n_queued = int(s->queue.size());
            if (s->stop && s->active.empty()) return;
        }
        bool progress = false;
        // completions (in stream order within each lane)
        for (Lane& ln : s->lanes) {
            while (!ln.flight.empty()) {
                Flight f = ln.flight.front();
                const cudaError_t q = cudaEventQuery(f.ev);
                if (q == cudaErrorNotReady) break;
                if (q != cudaSuccess) {
                    cudaGetLastError();
                    fail_all(s, std::string("device error: ") + cudaGetErrorString(q));
                    return;
                }
                ln.flight.pop_front();
                s->ev_pool.push_back(f.ev);
                if (f.tc_wrote >= 0) s->tcache[size_t(f.tc_wrote)].add(f.l0, f.l1);
                if (f.last) finish(s, f.r);
                progress = true;
            }
        }
        // admission, first come first served
        while (!s->queue.empty() && admit(s, s->queue.front()) != Admit::kNoRoom) {
            s->queue.pop_front();
            progress = true;
        }
        s->n_queued = int(s->queue.size());
        // issue: the admitted request with the least remaining work over all
        // lanes (its own lane having room), while fewer chunks than lanes
        // are in flight.  Step-two kernels fill the GPU, so chunks of
        // different lanes mostly run one after the other: choosing over all
        // lanes lets a large request run at the GPU's full rate when nothing
        // smaller waits, instead of sharing it with the other lanes' work.
        {
            int total = 0;
            for (const Lane& ln : s->lanes) total += int(ln.flight.size());
            const int cap = int(s->lanes.size());
            const int pol = s->cfg.policy;
            // XS_POLICY_DEADLINE: the request whose deadline -- submission
            // plus its remaining work at kDeadlineRate -- comes first
            auto key = [&](const Request* r) {
                if (pol == XS_POLICY_ROUND_ROBIN) return double(r->last_issue);
                if (pol == XS_POLICY_DEADLINE)
                    return std::chrono::duration<double, std::milli>(r->t_submit.time_since_epoch()).count() +
                           r->remaining / kDeadlineRate;
                return r->remaining;
            };
            while (total < cap) {
                Request* best = nullptr;
                double best_key = 0.0;
                for (Request* r : s->active)
                    if (r->next < r->chunks.size() && int(s->lanes[size_t(r->lane)].flight.size()) < depth) {
                        const double k = key(r);
                        if (!best || k < best_key) {
                            best = r;
                            best_key = k;
                        }
                    }
                if (!best) break;
                best->last_issue = ++s->issue_seq;
                if (!issue(s, best)) {
                    cudaGetLastError();
                    fail_all(s, std::string("launch failed: ") + xs_last_error());
                    return;
                }
                ++total;
                progress = true;
            }
        }
        if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

// Q(T) of a molecule from its states, computed on the device once per T.
int molecule_partition(xs_server* s, int mol, double temperature, double* q) {
    std::lock_guard<std::mutex> lk(s->qmu);
    Molecule& m = s->mols[size_t(mol)];
    if (!m.d_se)
        return sfail(XS_ERR_INVALID, "xs_server_submit: partition <= 0 needs the molecule's states "
                                     "(xs_server_add_states)");
    auto it = m.qcache.find(temperature);
    if (it != m.qcache.end()) {
        *q = it->second;
        return XS_OK;
    }
    DevGuard dg(s->device);
    const double beta = xs::partition_beta(temperature);
    double* d_beta = s->d_pwork;
    double* d_q = s->d_pwork + 1;
    double* work = s->d_pwork + 2;
    cudaError_t err = cudaMemcpyAsync(d_beta, &beta, sizeof(double), cudaMemcpyHostToDevice, s->aux);
    if (err == cudaSuccess) err = xs::partition_on_stream(m.d_se, m.d_sg, long(m.ns), d_beta, 1, d_q, work, s->aux);
    double val = 0.0;
    if (err == cudaSuccess) err = cudaMemcpyAsync(&val, d_q, sizeof(double), cudaMemcpyDeviceToHost, s->aux);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s->aux);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return sfail(XS_ERR_CUDA, std::string("partition function: ") + cudaGetErrorString(err));
    }
    if (m.qcache.size() > 4096) m.qcache.clear();
    m.qcache[temperature] = val;
    *q = val;
    return XS_OK;
}

}  // namespace

extern "C" {

int xs_server_create(int device, const xs_server_config* cfg, xs_server** out) {
    if (!out) return sfail(XS_ERR_INVALID, "xs_server_create: out is NULL");
    *out = nullptr;
    xs_server_config c{};
    if (cfg) c = *cfg;
    if (c.lanes <= 0) c.lanes = 4;
    if (c.depth <= 0) c.depth = 2;
    if (!(c.chunk_pairs > 0.0)) c.chunk_pairs = 4.0e9;
    if (c.chunk_lines == 0) c.chunk_lines = size_t(1) << 22;
    if (c.host_budget == 0) c.host_budget = size_t(1) << 30;
    if (c.lanes > 16 || c.depth > 8) return sfail(XS_ERR_INVALID, "xs_server_create: lanes <= 16, depth <= 8");
    if (c.policy != XS_POLICY_LEAST_WORK && c.policy != XS_POLICY_ROUND_ROBIN && c.policy != XS_POLICY_DEADLINE)
        return sfail(XS_ERR_INVALID, "xs_server_create: unknown policy");
    if (c.tcache_bytes == 0) c.tcache_bytes = 4LL << 30;
    auto* s = new xs_server();
    s->device = device;
    s->cfg = c;
    s->mols.reserve(kMaxMolecules);
    DevGuard dg(device);
    // lanes: a stream and an engine each, scratch sized for the largest chunk
    xs_options o{};
    o.profile = XS_VOIGT;
    o.precision = XS_FP64;
    size_t scratch = xs_scratch_bytes_needed(&o, 1, c.chunk_lines);
    o.precision = XS_MIXED;
    scratch = std::max(scratch, xs_scratch_bytes_needed(&o, 1, c.chunk_lines));
    scratch = ((scratch + 255) & ~size_t(255)) + (size_t(64) << 20);  // + the line-split parts
    for (int k = 0; k < c.lanes; ++k) {
        Lane ln;
        int rc = xs_engine_create(device, &ln.eng);
        if (rc == XS_OK && cudaStreamCreateWithFlags(&ln.st, cudaStreamNonBlocking) != cudaSuccess)
            rc = sfail(XS_ERR_CUDA, "cudaStreamCreate");
        if (rc == XS_OK) rc = xs_engine_set_stream(ln.eng, ln.st);
        if (rc == XS_OK) rc = xs::engine_reserve(ln.eng, scratch);
        if (rc != XS_OK) {
            if (ln.eng) xs_engine_destroy(ln.eng);
            if (ln.st) cudaStreamDestroy(ln.st);
            for (Lane& l : s->lanes) {
                xs_engine_destroy(l.eng);
                cudaStreamDestroy(l.st);
            }
            delete s;
            return rc;
        }
        s->lanes.push_back(ln);
    }
    s->resident = scratch * size_t(c.lanes) + (size_t(4) << 20) * size_t(c.lanes);
    if (c.device_budget == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        s->cfg.device_budget = fr > (size_t(2) << 30) ? fr - (size_t(2) << 30) : fr / 2;
        s->cfg.device_budget += s->resident;
    }
    if (s->resident > s->cfg.device_budget) {
        for (Lane& l : s->lanes) {
            xs_engine_destroy(l.eng);
            cudaStreamDestroy(l.st);
        }
        delete s;
        return sfail(XS_ERR_NOMEM, "xs_server_create: the lanes' scratch alone exceeds device_budget");
    }
    // keep freed request memory in the pool instead of returning it
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        unsigned long long thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    if (!s->arena.init(c.host_budget)) {
        for (Lane& l : s->lanes) {
            xs_engine_destroy(l.eng);
            cudaStreamDestroy(l.st);
        }
        delete s;
        return sfail(XS_ERR_NOMEM, "xs_server_create: pinned host arena");
    }
    if (cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&s->d_pwork, (2 + xs::partition_work_doubles(1)) * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        if (s->aux) cudaStreamDestroy(s->aux);
        for (Lane& l : s->lanes) {
            xs_engine_destroy(l.eng);
            cudaStreamDestroy(l.st);
        }
        s->arena.release();
        delete s;
        return sfail(XS_ERR_NOMEM, "xs_server_create: partition work area");
    }
    s->worker = std::thread(scheduler, s);
    *out = s;
    return XS_OK;
}

int xs_server_destroy(xs_server* s) {
    if (!s) return XS_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    DevGuard dg(s->device);
    for (Lane& l : s->lanes) {
        cudaStreamSynchronize(l.st);
        for (Flight& f : l.flight) cudaEventDestroy(f.ev);
        xs_engine_destroy(l.eng);
        cudaStreamDestroy(l.st);
    }
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    for (TCache& e : s->tcache) cudaFree(e.s);
    if (s->aux) cudaStreamDestroy(s->aux);
    cudaFree(s->d_pwork);
    for (Molecule& m : s->mols) {
        cudaFree(m.d_se);
        cudaFree(m.d_sg);
        cudaFree(m.nu);
        cudaFree(m.e);
        cudaFree(m.a);
        cudaFree(m.g);
        cudaFree(m.nx);
        cudaFree(m.gns);
    }
    for (auto& kv : s->all) delete kv.second;
    s->arena.release();
    delete s;
    return XS_OK;
}

int xs_server_add_molecule(xs_server* s, const double* nu, const double* energies,
                           const double* aif, const int* gns, const double* gamma,
                           const double* n, size_t count, double mean_mass, double ref_temp,
                           int* molecule_id) {
    if (!s || !nu || !energies || !aif || !gns || !gamma || !n || !molecule_id || count == 0)
        return sfail(XS_ERR_INVALID, "xs_server_add_molecule: NULL argument or no lines");
    if (!(mean_mass > 0.0) || !(ref_temp > 0.0))
        return sfail(XS_ERR_INVALID, "xs_server_add_molecule: mass and reference temperature must be > 0");
    for (size_t i = 1; i < count; ++i)
        if (nu[i] < nu[i - 1])
            return sfail(XS_ERR_UNSORTED, "xs_server_add_molecule: line centres must be ascending");
    const size_t bytes = count * (5 * sizeof(double) + sizeof(int));
    DevGuard dg(s->device);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->resident + s->dev_requests + bytes > s->cfg.device_budget)
        return sfail(XS_ERR_NOMEM, "xs_server_add_molecule: over the device budget");
    if (s->mols.size() >= kMaxMolecules)
        return sfail(XS_ERR_INVALID, "xs_server_add_molecule: at most 64 molecules per server");
    Molecule m;
    m.n = count;
    m.mass = mean_mass;
    m.ref_temp = ref_temp;
    m.bytes = bytes;
    cudaError_t err = cudaSuccess;
    auto put = [&](double** dst, const double* src) {
        if (err == cudaSuccess) err = cudaMalloc(dst, count * sizeof(double));
        if (err == cudaSuccess) err = cudaMemcpy(*dst, src, count * sizeof(double), cudaMemcpyHostToDevice);
    };
    put(&m.nu, nu);
    put(&m.e, energies);
    put(&m.a, aif);
    put(&m.g, gamma);
    put(&m.nx, n);
    if (err == cudaSuccess) err = cudaMalloc(&m.gns, count * sizeof(int));
    if (err == cudaSuccess) err = cudaMemcpy(m.gns, gns, count * sizeof(int), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) {
        cudaGetLastError();
        cudaFree(m.nu);
        cudaFree(m.e);
        cudaFree(m.a);
        cudaFree(m.g);
        cudaFree(m.nx);
        cudaFree(m.gns);
        return sfail(err == cudaErrorMemoryAllocation ? XS_ERR_NOMEM : XS_ERR_CUDA,
                     std::string("xs_server_add_molecule: ") + cudaGetErrorString(err));
    }
    m.h_nu.assign(nu, nu + count);
    m.h_cum.resize(count + 1);
    m.h_cum[0] = 0.0;
    for (size_t i = 0; i < count; ++i) m.h_cum[i + 1] = m.h_cum[i] + nu[i];
    s->resident += bytes;
    *molecule_id = int(s->mols.size());
    s->mols.push_back(std::move(m));
    return XS_OK;
}

int xs_server_add_states(xs_server* s, int molecule_id, const double* energies, const int* gns,
                         size_t count) {
    if (!s || !energies || !gns || count == 0)
        return sfail(XS_ERR_INVALID, "xs_server_add_states: NULL argument or no states");
    DevGuard dg(s->device);
    std::lock_guard<std::mutex> lk(s->mu);
    std::lock_guard<std::mutex> lq(s->qmu);
    if (molecule_id < 0 || size_t(molecule_id) >= s->mols.size())
        return sfail(XS_ERR_INVALID, "xs_server_add_states: no such molecule");
    Molecule& m = s->mols[size_t(molecule_id)];
    const size_t bytes = count * (sizeof(double) + sizeof(int));
    if (s->resident + s->dev_requests + bytes > s->cfg.device_budget)
        return sfail(XS_ERR_NOMEM, "xs_server_add_states: over the device budget");
    double* de = nullptr;
    int* dg2 = nullptr;
    cudaError_t err = cudaMalloc(&de, count * sizeof(double));
    if (err == cudaSuccess) err = cudaMalloc(&dg2, count * sizeof(int));
    if (err == cudaSuccess) err = cudaMemcpy(de, energies, count * sizeof(double), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dg2, gns, count * sizeof(int), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) {
        cudaGetLastError();
        cudaFree(de);
        cudaFree(dg2);
        return sfail(XS_ERR_CUDA, std::string("xs_server_add_states: ") + cudaGetErrorString(err));
    }
    cudaFree(m.d_se);
    cudaFree(m.d_sg);
    m.d_se = de;
    m.d_sg = dg2;
    m.ns = count;
    m.qcache.clear();
    s->resident += bytes;
    return XS_OK;
}

int xs_server_submit(xs_server* s, const xs_request* q, unsigned long long* request_id) {
    if (!s || !q || !request_id) return sfail(XS_ERR_INVALID, "xs_server_submit: NULL argument");
    const auto t0 = Clock::now();
    *request_id = 0;
    int nmol;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->fatal.empty()) return sfail(XS_ERR_CUDA, "server stopped: " + s->fatal);
        nmol = int(s->mols.size());
    }
    if (q->molecule < 0 || q->molecule >= nmol) return sfail(XS_ERR_INVALID, "xs_server_submit: no such molecule");
    if (q->profile != XS_VOIGT && q->profile != XS_DOPPLER)
        return sfail(XS_ERR_UNSUPPORTED, "xs_server_submit: profile must be VOIGT or DOPPLER");
    if (q->precision != XS_FP64 && q->precision != XS_MIXED)
        return sfail(XS_ERR_INVALID, "xs_server_submit: precision");
    if (!(q->temperature > 0.0) || !(q->df > 0.0) || q->npoints < 1 || !(q->pressure > 0.0))
        return sfail(XS_ERR_INVALID, "xs_server_submit: T, P and df must be > 0, npoints >= 1");
    double partition = q->partition;
    if (!(partition > 0.0)) {
        const int rc = molecule_partition(s, q->molecule, q->temperature, &partition);
        if (rc != XS_OK) return rc;
    }
    auto* r = new Request();
    r->q = *q;
    r->q.partition = partition;
    const Molecule& m = s->mols[size_t(q->molecule)];
    r->opt.profile = q->profile;
    r->opt.convention = XS_CONV_GPU;
    r->opt.precision = q->precision;
    r->opt.cpu_threads = 1;
    r->opt.mean_mass = m.mass;
    r->opt.ref_temp = m.ref_temp;
    r->opt.half_width = 0.1;
    r->opt.dfreq = q->df;
    r->cond.temperature = q->temperature;
    r->cond.partition = partition;
    r->cond.pressure = q->pressure;
    r->cond.gamma_scale = q->pressure;
    r->cond.cut = q->cut;
    const double cut = q->cut > 0.0 ? q->cut
                                     : (q->profile == XS_VOIGT ? std::fmin(25.0 * q->pressure, 100.0) : 100.0);
    // Doppler pairs beyond ~6 Doppler widths add exactly 0 and are skipped
    // (the erf saturation of step one), so their work is counted over that
    // span: nu_max * 6 sqrt(2 k T N_A / M) / c plus the bin and a margin.
    double cost_cut = cut;
    if (q->profile == XS_DOPPLER) {
        const double kB = 1.380658e-16, NA = 6.0221412927e23, c = 2.99792458e10;
        const double nu_max = q->f0 + double(q->npoints) * q->df + cut;
        const double w = 6.0 * std::sqrt(2.0 * kB * q->temperature * NA / m.mass) / c;
        cost_cut = std::fmin(cut, std::fabs(nu_max) * w * 1.01 + 2.5 * q->df);
    }
    plan_chunks(m.index(), q->f0, q->df, q->npoints, cut, cost_cut, s->cfg.chunk_pairs,
                s->cfg.chunk_lines, r->chunks);
    for (const ChunkPlan& c : r->chunks) {
        if (c.l1 - c.l0 > s->cfg.chunk_lines) {
            delete r;
            return sfail(XS_ERR_NOMEM, "xs_server_submit: a single 256-point tile needs more lines "
                                       "than chunk_lines");
        }
        r->pairs += c.pairs;
        r->remaining += c.cost;
    }
    r->lines = m.index().upper(q->f0 + double(q->npoints - 1) * q->df + cut) -
               m.index().lower(q->f0 - cut);
    r->dev_bytes = request_device_bytes(*q);
    if (s->resident + r->dev_bytes > s->cfg.device_budget ||
        sizeof(double) * size_t(q->npoints) + 256 > s->arena.size()) {
        delete r;
        return sfail(XS_ERR_NOMEM, "xs_server_submit: the request alone exceeds the memory budget");
    }
    r->t_submit = t0;
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    s->all[r->id] = r;
    s->incoming.push_back(r);
    s->cv_work.notify_all();
    *request_id = r->id;
    return XS_OK;
}

int xs_server_wait(xs_server* s, unsigned long long id, double* out, int npoints,
                   xs_request_info* info, int timeout_ms) {
    if (!s) return sfail(XS_ERR_INVALID, "xs_server_wait: NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return sfail(XS_ERR_INVALID, "xs_server_wait: unknown request id");
    Request* r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
        return sfail(XS_ERR_TIMEOUT, "xs_server_wait: not finished yet");
    if (info) {
        info->status = r->status;
        info->latency_ms = ms_between(r->t_submit, r->t_done);
        info->queue_ms = r->t_admit.time_since_epoch().count() ? ms_between(r->t_submit, r->t_admit) : 0.0;
        info->run_ms = r->t_admit.time_since_epoch().count() ? ms_between(r->t_admit, r->t_done) : 0.0;
        info->chunks = int(r->chunks.size());
        info->line_evals = r->pairs;
        info->lines = r->lines;
        info->err_bound = xs_error_bound(r->opt.profile, r->opt.precision);
        info->tcache_chunks = r->tc_chunks;
    }
    int rc = r->status;
    std::string err = r->error;
    if (rc == XS_OK && out) {
        if (npoints != r->q.npoints) {
            rc = XS_ERR_INVALID;
            err = "xs_server_wait: npoints differs from the request's";
        } else {
            std::memcpy(out, s->arena.at(r->host_off), sizeof(double) * size_t(npoints));
        }
    }
    if (r->host_off != SIZE_MAX) s->arena.free(r->host_off, r->host_bytes);
    s->all.erase(it);
    delete r;
    if (rc != XS_OK) return sfail(rc, err.empty() ? "request failed" : err);
    return XS_OK;
}

int xs_server_pending(xs_server* s, int* queued, int* active) {
    if (!s) return sfail(XS_ERR_INVALID, "xs_server_pending: NULL server");
    if (queued) *queued = s->n_queued;
    if (active) *active = s->n_active;
    return XS_OK;
}

int xs_plan_chunks(const double* nu, size_t n, double f0, double df, int npoints, double cut,
                   double max_pairs, size_t max_lines, int cap, int* start, int* points,
                   size_t* l0, size_t* l1, double* pairs, int* nchunks) {
    if ((!nu && n) || !nchunks || npoints < 1 || !(df > 0.0) || !(cut > 0.0) || !(max_pairs > 0.0))
        return sfail(XS_ERR_INVALID, "xs_plan_chunks: bad arguments");
    for (size_t i = 1; i < n; ++i)
        if (nu[i] < nu[i - 1]) return sfail(XS_ERR_UNSORTED, "xs_plan_chunks: nu must be ascending");
    std::vector<double> cum(n + 1, 0.0);
    for (size_t i = 0; i < n; ++i) cum[i + 1] = cum[i] + nu[i];
    LineIndex L;
    L.nu = nu;
    L.cum = cum.data();
    L.n = n;
    std::vector<ChunkPlan> plan;
    plan_chunks(L, f0, df, npoints, cut, cut, max_pairs, max_lines ? max_lines : SIZE_MAX, plan);
    *nchunks = int(plan.size());
    if (int(plan.size()) > cap) return sfail(XS_ERR_INVALID, "xs_plan_chunks: more chunks than cap");
    for (size_t k = 0; k < plan.size(); ++k) {
        if (start) start[k] = plan[k].start;
        if (points) points[k] = plan[k].points;
        if (l0) l0[k] = plan[k].l0;
        if (l1) l1[k] = plan[k].l1;
        if (pairs) pairs[k] = plan[k].pairs;
    }
    return XS_OK;
}

int xs_split_grid(const double* nu, size_t n, double f0, double df, int npoints, double cut,
                  int nranks, int rank, int* start, int* points, size_t* l0, size_t* l1,
                  double* pairs) {
    if ((!nu && n) || npoints < 1 || !(df > 0.0) || !(cut > 0.0) || nranks < 1 || rank < 0 ||
        rank >= nranks || !start || !points || !l0 || !l1)
        return sfail(XS_ERR_INVALID, "xs_split_grid: bad arguments");
    for (size_t i = 1; i < n; ++i)
        if (nu[i] < nu[i - 1]) return sfail(XS_ERR_UNSORTED, "xs_split_grid: nu must be ascending");
    std::vector<double> cum(n + 1, 0.0);
    for (size_t i = 0; i < n; ++i) cum[i + 1] = cum[i] + nu[i];
    LineIndex L;
    L.nu = nu;
    L.cum = cum.data();
    L.n = n;
    // one plan entry per 256-point tile (a limit no tile fits in)
    std::vector<ChunkPlan> tiles;
    plan_chunks(L, f0, df, npoints, cut, cut, 1e-300, SIZE_MAX, tiles);
    const int nt = int(tiles.size());
    std::vector<double> acc(size_t(nt) + 1, 0.0);
    for (int t = 0; t < nt; ++t) acc[size_t(t) + 1] = acc[size_t(t)] + tiles[size_t(t)].pairs;
    // rank k starts at the first tile whose preceding work reaches k / nranks
    // of the total (rank 0 at tile 0, the end at the last tile)
    auto boundary = [&](int k) {
        if (k <= 0) return 0;
        if (k >= nranks) return nt;
        const double want = acc[size_t(nt)] * double(k) / double(nranks);
        return int(std::lower_bound(acc.begin(), acc.end(), want) - acc.begin());
    };
    int tb = boundary(rank), te = boundary(rank + 1);
    if (te < tb) te = tb;
    if (tb >= nt || te == tb) {
        *start = tb < nt ? tiles[size_t(tb)].start : npoints;
        *points = 0;
        *l0 = *l1 = 0;
        if (pairs) *pairs = 0.0;
        return XS_OK;
    }
    *start = tiles[size_t(tb)].start;
    *points = tiles[size_t(te) - 1].start + tiles[size_t(te) - 1].points - *start;
    *l0 = tiles[size_t(tb)].l0;
    *l1 = tiles[size_t(te) - 1].l1;
    if (pairs) *pairs = acc[size_t(te)] - acc[size_t(tb)];
    return XS_OK;
}

}  // extern "C"
