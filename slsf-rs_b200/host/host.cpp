/*
 * Host layer above the C ABI (include/slsf_host.h): the C++ restatement of
 * the parts of SLSF-rs's Rust host that drive the hot path -- ThetaModel's
 * MonteCarlo methods and carlo-mc's binning (src/model.rs:308-477, :857-934),
 * the task expansion's seed formula and disorder draw (src/model.rs:697-810,
 * src/initialization.rs:5-31) -- and a continuous-batching server.  Every
 * device operation goes through slsf_gpu.h.
 */
#include "../../include/slsf_host.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <list>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

thread_local std::string g_host_error;

int fail(int code, const std::string& msg) {
    g_host_error = msg;
    return code;
}

/* Copies the GPU library's message after a failed ABI call. */
int gpu_fail(int code) {
    char buf[512];
    slsf_last_error(buf, sizeof(buf));
    g_host_error = buf;
    return code;
}

#define HOST_TRY(call)                    \
    do {                                  \
        int rc_ = (call);                 \
        if (rc_ != SLSF_OK) return gpu_fail(rc_); \
    } while (0)

/* FastRng (src/types.rs:16-82): SplitMix64 words; rand's bool is the sign of
 * the low 32-bit word. */
struct FastRng {
    uint64_t state;
    explicit FastRng(uint64_t seed) : state(seed) {}
    uint64_t next() {
        state += 0x9E3779B97F4A7C15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    bool boolean() { return (int32_t)(uint32_t)next() < 0; }
};

/* initialize_two_point_layer_disorder (src/initialization.rs:5-31). */
int two_point(double* values, size_t n, double mean, double delta, FastRng& rng, const char* name) {
    if (delta < 0.0) return fail(SLSF_ERR_INVALID, std::string("\xce\xb4") + name + " must be nonnegative");
    const double lower = mean - delta, upper = mean + delta;
    if (lower < 0.0)
        return fail(SLSF_ERR_INVALID, std::string("two-point layer disorder requires ") + name + "_mean - \xce\xb4" +
                                          name + " >= 0");
    for (size_t i = 0; i < n; ++i) values[i] = delta == 0.0 ? mean : (rng.boolean() ? upper : lower);
    return SLSF_OK;
}

double mean_of(const double* x, size_t n, size_t stride) {
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += x[i * stride];
    return s / (double)n;
}

double now_s(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

size_t slsf_host_last_error(char* buf, size_t len) {
    if (buf && len) {
        const size_t n = std::min(len - 1, g_host_error.size());
        std::memcpy(buf, g_host_error.data(), n);
        buf[n] = '\0';
    }
    return g_host_error.size();
}

int slsf_binned_estimate(const double* samples, size_t n, size_t binsize, double* mean, double* stderr_out,
                         size_t* n_bins) {
    if (binsize == 0 || binsize > n) return fail(SLSF_ERR_INVALID, "binsize is larger than the sample series");
    const size_t nb = n / binsize;
    std::vector<double> b(nb);
    for (size_t k = 0; k < nb; ++k) b[k] = mean_of(samples + k * binsize, binsize, 1);
    const double m = mean_of(b.data(), nb, 1);
    double v = 0;
    for (double x : b) v += (x - m) * (x - m);
    if (mean) *mean = m;
    if (stderr_out) *stderr_out = nb > 1 ? std::sqrt(v / (double)(nb - 1)) / std::sqrt((double)nb) : 0.0;
    if (n_bins) *n_bins = nb;
    return SLSF_OK;
}

int slsf_estimates_from_bins(const double* bm, size_t nb, double volume, double beta, slsf_estimates* out) {
    if (!bm || !out || nb == 0) return fail(SLSF_ERR_INVALID, "no bins");
    constexpr int C = SLSF_BIN_COLS;
    std::memset(out, 0, sizeof(*out));
    out->n_bins = (uint32_t)nb;
    double total[C] = {0};
    for (size_t k = 0; k < nb; ++k)
        for (int c = 0; c < C; ++c) total[c] += bm[k * C + c];
    for (int c = 0; c < C; ++c) {
        out->mean[c] = total[c] / (double)nb;
        double v = 0;
        for (size_t k = 0; k < nb; ++k) v += (bm[k * C + c] - out->mean[c]) * (bm[k * C + c] - out->mean[c]);
        out->err[c] = nb > 1 ? std::sqrt(v / (double)(nb - 1)) / std::sqrt((double)nb) : 0.0;
    }
    /* register_theta_evaluables (src/model.rs:857-888) */
    auto eval = [&](const double* c, double r[SLSF_DERIVED]) {
        r[0] = std::sqrt(c[2]);
        r[1] = beta * volume * c[2];
        r[2] = beta * beta * volume * (c[1] - c[0] * c[0]);
        const double rx = c[3] / volume - beta * (c[9] - c[6] * c[6]) / volume;
        const double ry = c[4] / volume - beta * (c[10] - c[7] * c[7]) / volume;
        r[3] = (rx + ry) / 2.0;
        r[4] = c[5] / volume - beta * (c[11] - c[8] * c[8]) / volume;
    };
    eval(out->mean, out->derived);
    if (nb > 1) {
        /* delete-one jackknife over bins */
        std::vector<double> jk(nb * SLSF_DERIVED);
        double jm[SLSF_DERIVED] = {0};
        for (size_t k = 0; k < nb; ++k) {
            double loo[C];
            for (int c = 0; c < C; ++c) loo[c] = (total[c] - bm[k * C + c]) / (double)(nb - 1);
            eval(loo, &jk[k * SLSF_DERIVED]);
            for (int q = 0; q < SLSF_DERIVED; ++q) jm[q] += jk[k * SLSF_DERIVED + q] / (double)nb;
        }
        for (int q = 0; q < SLSF_DERIVED; ++q) {
            double v = 0;
            for (size_t k = 0; k < nb; ++k) v += (jk[k * SLSF_DERIVED + q] - jm[q]) * (jk[k * SLSF_DERIVED + q] - jm[q]);
            out->derived_err[q] = std::sqrt(v * (double)(nb - 1) / (double)nb);
        }
    }
    return SLSF_OK;
}

uint64_t slsf_task_seed(uint64_t base, uint32_t l_z, uint32_t sample, double temperature, double djxy, double djz) {
    /* f64::round rounds halves away from zero; `as u64` saturates (NaN and
     * negatives to 0, values past the range to 2^64 - 1) */
    auto r = [](double x) -> uint64_t {
        const double v = std::round(x);
        if (!(v > 0.0)) return 0;
        if (v >= 18446744073709551616.0) return UINT64_MAX;
        return (uint64_t)v;
    };
    return base + 100000ull * l_z + 1000ull * sample + r(100.0 * temperature) + r(1000.0 * djxy) * 10000ull +
           r(1000.0 * djz);
}

int slsf_task_couplings(const slsf_theta_task* t, double* j_xy, double* j_z) {
    if (!t || !j_xy || !j_z) return fail(SLSF_ERR_INVALID, "NULL argument");
    FastRng rng(t->disorder_seed);
    if (t->j_xy_array) {
        std::memcpy(j_xy, t->j_xy_array, sizeof(double) * t->lz);
    } else if (int rc = two_point(j_xy, t->lz, t->j_xy, t->delta_j_xy, rng, "J_xy")) {
        return rc;
    }
    if (t->j_z_array) {
        std::memcpy(j_z, t->j_z_array, sizeof(double) * t->lz);
    } else if (int rc = two_point(j_z, t->lz, t->j_z_mean, t->delta_j_z, rng, "J_z")) {
        return rc;
    }
    for (uint32_t z = 0; z < t->lz; ++z)
        if (j_xy[z] < 0.0 || j_z[z] < 0.0)
            return fail(SLSF_ERR_INVALID, "theta simulation requires nonnegative layer couplings");
    return SLSF_OK;
}

int slsf_model_run(slsf_ctx* ctx, const slsf_theta_task* t, int batched, slsf_estimates* out) {
    if (!ctx || !t || !out) return fail(SLSF_ERR_INVALID, "NULL argument");
    if (t->binsize == 0) return fail(SLSF_ERR_INVALID, "binsize must be positive");
    if (t->sweeps < t->binsize) return fail(SLSF_ERR_INVALID, "sweeps must be at least binsize");
    std::vector<double> jx(t->lz ? t->lz : 1), jz(t->lz ? t->lz : 1);
    if (t->lz && slsf_task_couplings(t, jx.data(), jz.data())) return SLSF_ERR_INVALID;
    const uint32_t nb = t->sweeps / t->binsize;
    slsf_task_desc d = {};
    d.lx = t->lx;
    d.ly = t->ly;
    d.lz = t->lz;
    d.temperature = t->temperature;
    d.proposal_width = t->proposal_width;
    d.wolff_steps = t->wolff_steps;
    d.seed = t->seed;
    d.j_xy = jx.data();
    d.n_j_xy = t->lz;
    d.j_z = jz.data();
    d.n_j_z = t->lz;
    d.thermalization = t->thermalization;
    d.binsize = t->binsize;
    d.n_bins = batched ? nb : 0;
    slsf_task* task = nullptr;
    HOST_TRY(slsf_task_create(ctx, &d, &task));
    struct Guard {
        slsf_task* t;
        ~Guard() { slsf_task_destroy(t); }
    } guard{task};
    /* ThetaModel::init (src/model.rs:373-377) */
    HOST_TRY(slsf_task_init_random(task));
    const double volume = (double)t->lx * t->ly * t->lz;
    const double beta = 1.0 / t->temperature;
    std::vector<double> bins((size_t)nb * SLSF_BIN_COLS, 0.0);
    uint64_t accepted = 0;
    if (batched) {
        slsf_sweep_stats st = {};
        HOST_TRY(slsf_batch_run(ctx, &task, 1, t->thermalization + t->sweeps, &st));
        accepted = st.accepted;
        uint64_t m = 0;
        HOST_TRY(slsf_task_get_bins(task, bins.data(), nb, &m));
        out->measurements = m;
    } else {
        /* carlo-mc's schedule: thermalization sweeps, then sweep + measure */
        slsf_sweep_stats st = {};
        if (t->thermalization) {
            HOST_TRY(slsf_task_sweep(task, t->thermalization, &st));
            accepted += st.accepted;
        }
        std::vector<double> row(SLSF_BIN_COLS);
        for (uint32_t s = 0; s < nb * t->binsize; ++s) {
            HOST_TRY(slsf_task_sweep(task, 1, &st));
            accepted += st.accepted;
            slsf_observables o;
            HOST_TRY(slsf_task_measure(task, &o));
            /* ThetaModel::measure's stream (src/model.rs:406-409, :890-904) */
            const double r[SLSF_BIN_COLS] = {o.energy, o.energy * o.energy, o.magnetization_squared,
                                             o.cos_x, o.cos_y, o.cos_z, o.sin_x, o.sin_y, o.sin_z,
                                             o.sin_x * o.sin_x, o.sin_y * o.sin_y, o.sin_z * o.sin_z};
            double* b = &bins[(size_t)(s / t->binsize) * SLSF_BIN_COLS];
            for (int c = 0; c < SLSF_BIN_COLS; ++c) b[c] += r[c] / (double)t->binsize;
        }
        for (uint32_t s = nb * t->binsize; s < t->sweeps; ++s) HOST_TRY(slsf_task_sweep(task, 1, &st));
        out->measurements = (uint64_t)nb * t->binsize;
    }
    const uint64_t m = out->measurements;
    if (int rc = slsf_estimates_from_bins(bins.data(), nb, volume, beta, out)) return rc;
    out->measurements = m;
    out->acceptance = (double)accepted / (volume * (double)(t->thermalization + t->sweeps));
    return SLSF_OK;
}

}  // extern "C"

/* ---------------------------------------------------------------- server */

struct Pending {
    slsf_request req;
    std::vector<double> jxy, jz;
    double submit_s;
    uint32_t bypassed = 0;
    /* restored from a checkpoint while running: the task's device state,
     * its bin plan and its progress */
    std::vector<char> state;
    uint32_t plan_binsize = 0, plan_n_bins = 0, remaining = 0;
    uint64_t accepted = 0, cluster_sites = 0;
};

struct Active {
    Pending p;
    slsf_task* task = nullptr;
    uint64_t bytes = 0;
    uint32_t remaining = 0;
    uint32_t binsize = 1;
    uint32_t n_bins = 0;
    double admit_s = 0;
    uint64_t accepted = 0;
    uint64_t cluster_sites = 0;
    bool cancelled = false;
};

struct slsf_server {
    slsf_ctx* ctx = nullptr;
    slsf_server_config cfg = {};
    std::unordered_map<uint64_t, std::vector<double>> kept_bins; /* guarded by mu */
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;                /* guards queue, results, cancel set, stats */
    std::condition_variable cv;   /* new work or stop */
    std::condition_variable idle; /* queue and active set empty */
    std::list<Pending> queue; /* stable iterators: submissions append while admission scans */
    std::vector<slsf_result> results;
    std::unordered_set<uint64_t> cancel;
    slsf_server_stats stats = {};
    /* owned by whichever thread runs epochs */
    std::vector<Active> active;
    uint64_t used = 0;
    std::atomic<bool> stop{false};
    std::atomic<bool> running{false};
    std::thread worker;
    std::atomic<uint32_t> n_active{0};
    uint32_t admitting = 0; /* requests between the queue and the active set (guarded by mu) */
    std::vector<uint64_t> admitting_tags;
    std::string worker_error; /* set when the worker stopped on a device error */
};

namespace {

slsf_result make_result(const Pending& p, int status, const std::string& msg, double now) {
    slsf_result r;
    std::memset(&r, 0, sizeof(r));
    r.tag = p.req.tag;
    r.status = status;
    std::strncpy(r.message, msg.c_str(), sizeof(r.message) - 1);
    r.submit_s = p.submit_s;
    r.admit_s = now;
    r.finish_s = now;
    return r;
}

/* The checks a sweep makes (ThetaLattice::new, ThetaModel::new, the
 * red-black sweep and the proposal, src/types.rs:120-129, src/model.rs:318-348,
 * src/updates.rs), made at submission so that a bad request fails alone
 * instead of failing the launch it would share. */
std::string validate(const Pending& p) {
    const slsf_request& r = p.req;
    if (r.lx == 0) return "L_x must be positive";
    if (r.ly == 0) return "L_y must be positive";
    if (r.lz == 0) return "L_z must be positive";
    if ((uint64_t)r.lx * r.ly * r.lz > (1ull << 31)) return "lattice volume exceeds 2^31 sites";
    if (p.jxy.size() != r.lz) return "J_xy_array length must match Lz";
    if (p.jz.size() != r.lz) return "J_z_array length must match Lz";
    for (uint32_t z = 0; z < r.lz; ++z)
        if (!(p.jxy[z] >= 0.0) || !(p.jz[z] >= 0.0)) return "theta simulation requires nonnegative layer couplings";
    if (!(r.temperature > 0.0) || !std::isfinite(r.temperature)) return "temperature T must be positive and finite";
    if (!(r.proposal_width >= 0.0) || !std::isfinite(r.proposal_width))
        return "proposal_width must be nonnegative and finite";
    if (r.lx % 2 || r.ly % 2 || r.lz % 2) return "red-black Metropolis sweep requires even lattice dimensions";
    if (r.sweeps == 0) return "sweeps must be positive";
    return "";
}

/* Admission: FIFO, but a request that does not fit may be passed by later
 * ones that do, at most 8 epochs in a row (then admission waits for it). */
void admit(slsf_server* s) {
    struct Pick {
        Pending p;
        uint64_t bytes;
        uint32_t binsize, n_bins;
        slsf_task* task;
        int rc;
        std::string msg;
    };
    const uint64_t budget = s->cfg.budget_bytes;
    std::vector<Pick> picks;
    {
        /* Choose under the lock; s->used and s->active change only on the
         * thread that runs epochs, which is this one. */
        std::lock_guard<std::mutex> lock(s->mu);
        uint64_t used = s->used;
        size_t n_active = s->active.size();
        for (auto it = s->queue.begin(); it != s->queue.end();) {
            if (s->cfg.max_active && n_active >= s->cfg.max_active) break;
            Pending& p = *it;
            const uint32_t measured = p.req.sweeps > p.req.thermalization ? p.req.sweeps - p.req.thermalization : 0;
            /* complete bins only (carlo drops a partial last bin) */
            uint32_t n_bins, binsize;
            if (!p.state.empty()) {
                binsize = p.plan_binsize;
                n_bins = p.plan_n_bins;
            } else if (p.req.binsize) {
                binsize = p.req.binsize;
                n_bins = std::max<uint32_t>(1, measured / binsize);
            } else {
                n_bins = std::max<uint32_t>(
                    1, std::min<uint32_t>(p.req.n_bins ? p.req.n_bins : 1, std::max<uint32_t>(measured, 1)));
                binsize = std::max<uint32_t>(1, measured / n_bins);
            }
            const uint64_t bytes = slsf_task_bytes(p.req.lx, p.req.ly, p.req.lz, n_bins);
            if (bytes > budget) {
                /* can never fit: reject now */
                s->results.push_back(make_result(p, SLSF_ERR_BUDGET,
                                                 "request does not fit in the server's device memory budget",
                                                 now_s(s->t0)));
                s->stats.failed++;
                it = s->queue.erase(it);
                continue;
            }
            if (used + bytes > budget) {
                /* later requests may pass a blocked head at most 8 epochs in a row */
                if (it == s->queue.begin() && ++p.bypassed > 8) break;
                ++it;
                continue;
            }
            s->admitting_tags.push_back(p.req.tag);
            picks.push_back(Pick{std::move(p), bytes, binsize, n_bins, nullptr, SLSF_OK, ""});
            it = s->queue.erase(it);
            used += bytes;
            ++n_active;
        }
        s->admitting += (uint32_t)picks.size();
    }
    /* Device set-up outside the lock: submissions continue meanwhile. */
    for (Pick& k : picks) {
        slsf_task_desc d = {};
        d.lx = k.p.req.lx;
        d.ly = k.p.req.ly;
        d.lz = k.p.req.lz;
        d.temperature = k.p.req.temperature;
        d.proposal_width = k.p.req.proposal_width;
        d.wolff_steps = k.p.req.wolff_steps;
        d.seed = k.p.req.seed;
        d.j_xy = k.p.jxy.data();
        d.n_j_xy = k.p.jxy.size();
        d.j_z = k.p.jz.data();
        d.n_j_z = k.p.jz.size();
        d.thermalization = k.p.req.thermalization;
        d.binsize = k.binsize;
        d.n_bins = k.n_bins;
        k.rc = slsf_task_create(s->ctx, &d, &k.task);
        if (k.rc == SLSF_OK)
            k.rc = k.p.state.empty() ? slsf_task_init_random(k.task)
                                     : slsf_task_state_load(k.task, k.p.state.data(), k.p.state.size(), nullptr);
        if (k.rc != SLSF_OK) {
            char buf[160];
            slsf_last_error(buf, sizeof(buf));
            k.msg = buf;
            if (k.task) slsf_task_destroy(k.task);
            k.task = nullptr;
        }
    }
    std::lock_guard<std::mutex> lock(s->mu);
    const double t = now_s(s->t0);
    s->admitting_tags.clear();
    for (Pick& k : picks) {
        s->admitting--;
        if (k.rc != SLSF_OK) {
            s->cancel.erase(k.p.req.tag);
            s->results.push_back(make_result(k.p, k.rc, k.msg, t));
            s->stats.failed++;
            continue;
        }
        Active a;
        a.p = std::move(k.p);
        a.task = k.task;
        a.bytes = k.bytes;
        a.remaining = a.p.state.empty() ? a.p.req.sweeps : a.p.remaining;
        a.accepted = a.p.accepted;
        a.cluster_sites = a.p.cluster_sites;
        a.p.state.clear();
        a.p.state.shrink_to_fit();
        a.binsize = k.binsize;
        a.n_bins = k.n_bins;
        a.admit_s = t;
        s->used += k.bytes;
        s->active.push_back(std::move(a));
    }
    s->stats.peak_active = std::max<uint64_t>(s->stats.peak_active, s->active.size());
    s->stats.peak_bytes = std::max<uint64_t>(s->stats.peak_bytes, s->used);
}

/* Retire finished or cancelled tasks: one gather of their bins, estimates,
 * results, memory back. */
int retire(slsf_server* s) {
    std::vector<size_t> done;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        for (size_t i = 0; i < s->active.size(); ++i) {
            Active& a = s->active[i];
            if (s->cancel.count(a.p.req.tag)) {
                a.cancelled = true;
                s->cancel.erase(a.p.req.tag);
            }
            if (a.remaining == 0 || a.cancelled) done.push_back(i);
        }
    }
    if (done.empty()) return SLSF_OK;
    std::vector<slsf_task*> tasks;
    for (size_t i : done)
        if (!s->active[i].cancelled) tasks.push_back(s->active[i].task);
    /* tasks keep different bin counts: gather each task's own rows */
    std::vector<uint64_t> meas(tasks.size());
    std::vector<std::vector<double>> per(tasks.size());
    {
        size_t k = 0;
        for (size_t i : done) {
            Active& a = s->active[i];
            if (a.cancelled) continue;
            per[k].resize((size_t)a.n_bins * SLSF_BIN_COLS);
            ++k;
        }
    }
    {
        /* group by bin count so each group is one gather */
        std::vector<size_t> idx(tasks.size());
        for (size_t k = 0; k < idx.size(); ++k) idx[k] = k;
        std::vector<uint32_t> nb(tasks.size());
        size_t k = 0;
        for (size_t i : done)
            if (!s->active[i].cancelled) nb[k++] = s->active[i].n_bins;
        std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return nb[a] < nb[b]; });
        for (size_t lo = 0; lo < idx.size();) {
            size_t hi = lo;
            while (hi < idx.size() && nb[idx[hi]] == nb[idx[lo]]) ++hi;
            std::vector<slsf_task*> group;
            for (size_t q = lo; q < hi; ++q) group.push_back(tasks[idx[q]]);
            const uint32_t r = nb[idx[lo]];
            std::vector<double> out((hi - lo) * (size_t)r * SLSF_BIN_COLS);
            std::vector<uint64_t> gm(hi - lo);
            int rc = slsf_batch_get_bins(s->ctx, group.data(), group.size(), r, out.data(), gm.data());
            if (rc != SLSF_OK) return gpu_fail(rc);
            for (size_t q = lo; q < hi; ++q) {
                std::copy(out.begin() + (q - lo) * r * SLSF_BIN_COLS, out.begin() + (q - lo + 1) * r * SLSF_BIN_COLS,
                          per[idx[q]].begin());
                meas[idx[q]] = gm[q - lo];
            }
            lo = hi;
        }
    }
    std::vector<slsf_result> out;
    std::vector<std::pair<uint64_t, std::vector<double>>> kept;
    size_t k = 0;
    const double t = now_s(s->t0);
    for (size_t i : done) {
        Active& a = s->active[i];
        slsf_result r = make_result(a.p, SLSF_OK, "", t);
        r.admit_s = a.admit_s;
        r.sweeps = a.p.req.sweeps - a.remaining;
        r.accepted = a.accepted;
        r.cluster_sites = a.cluster_sites;
        if (a.cancelled) {
            r.status = SLSF_ERR_STATE;
            std::strncpy(r.message, "cancelled", sizeof(r.message) - 1);
        } else {
            const double vol = (double)a.p.req.lx * a.p.req.ly * a.p.req.lz;
            const uint32_t full = (uint32_t)std::min<uint64_t>(a.n_bins, meas[k] / a.binsize);
            if (full > 0) slsf_estimates_from_bins(per[k].data(), full, vol, 1.0 / a.p.req.temperature, &r.est);
            if (s->cfg.keep_bins && full > 0) {
                per[k].resize((size_t)full * SLSF_BIN_COLS);
                kept.emplace_back(r.tag, std::move(per[k]));
            }
            r.est.measurements = meas[k];
            r.est.acceptance = (double)a.accepted / (vol * (double)std::max<uint64_t>(1, r.sweeps));
            ++k;
        }
        slsf_task_destroy(a.task);
        s->used -= a.bytes;
        out.push_back(r);
    }
    std::lock_guard<std::mutex> lock(s->mu);
    for (auto it = done.rbegin(); it != done.rend(); ++it) s->active.erase(s->active.begin() + *it);
    for (auto& kb : kept) s->kept_bins[kb.first] = std::move(kb.second);
    for (auto& r : out) {
        if (r.status == SLSF_OK)
            s->stats.completed++;
        else
            s->stats.cancelled++;
        s->results.push_back(r);
    }
    if (s->queue.empty() && s->active.empty()) s->idle.notify_all();
    return SLSF_OK;
}

void notify_if_idle(slsf_server* s) {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->queue.empty() && s->active.empty() && !s->admitting) s->idle.notify_all();
}

/* One epoch: retire cancelled tasks, admit, advance every active task by up
 * to epoch_sweeps in one launch, retire the tasks that finished. */
int epoch(slsf_server* s) {
    const auto t0 = std::chrono::steady_clock::now();
    if (int rc = retire(s)) return rc;
    admit(s);
    s->n_active = (uint32_t)s->active.size();
    if (s->active.empty()) {
        notify_if_idle(s);
        return SLSF_OK;
    }
    std::vector<slsf_task*> tasks(s->active.size());
    std::vector<uint32_t> sweeps(s->active.size());
    for (size_t i = 0; i < s->active.size(); ++i) {
        tasks[i] = s->active[i].task;
        sweeps[i] = std::min(s->active[i].remaining, s->cfg.epoch_sweeps);
    }
    std::vector<slsf_sweep_stats> st(tasks.size());
    int rc = slsf_batch_run_v(s->ctx, tasks.data(), tasks.size(), sweeps.data(), st.data());
    if (rc != SLSF_OK) return gpu_fail(rc);
    uint64_t updates = 0;
    for (size_t i = 0; i < s->active.size(); ++i) {
        Active& a = s->active[i];
        a.remaining -= sweeps[i];
        a.accepted += st[i].accepted;
        a.cluster_sites += st[i].wolff_cluster_sites;
        updates += (uint64_t)sweeps[i] * a.p.req.lx * a.p.req.ly * a.p.req.lz;
    }
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stats.epochs++;
        s->stats.launches++;
        s->stats.site_updates += updates;
    }
    rc = retire(s);
    std::lock_guard<std::mutex> lock(s->mu);
    s->stats.busy_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

}  // namespace

extern "C" {

int slsf_server_create(slsf_ctx* ctx, const slsf_server_config* cfg, slsf_server** out) {
    if (!ctx || !out) return fail(SLSF_ERR_INVALID, "NULL argument");
    slsf_server* s = new slsf_server;
    s->ctx = ctx;
    if (cfg) s->cfg = *cfg;
    if (!s->cfg.epoch_sweeps) s->cfg.epoch_sweeps = 100;
    uint64_t used = 0, budget = 0;
    slsf_ctx_memory(ctx, &used, &budget);
    if (!s->cfg.budget_bytes || s->cfg.budget_bytes > budget - used) s->cfg.budget_bytes = budget - used;
    s->t0 = std::chrono::steady_clock::now();
    *out = s;
    return SLSF_OK;
}

int slsf_server_stop(slsf_server* s) {
    if (!s) return fail(SLSF_ERR_INVALID, "NULL argument");
    if (s->running) {
        s->stop = true;
        s->cv.notify_all();
        s->worker.join();
        s->running = false;
        s->stop = false;
    }
    return SLSF_OK;
}

int slsf_server_destroy(slsf_server* s) {
    if (!s) return SLSF_OK;
    slsf_server_stop(s);
    for (Active& a : s->active) slsf_task_destroy(a.task);
    delete s;
    return SLSF_OK;
}

int slsf_server_submit(slsf_server* s, const slsf_request* r) {
    if (!s || !r) return fail(SLSF_ERR_INVALID, "NULL argument");
    Pending p;
    p.req = *r;
    const uint32_t lz = r->lz;
    if (lz && r->j_xy && r->j_z) {
        p.jxy.assign(r->j_xy, r->j_xy + lz);
        p.jz.assign(r->j_z, r->j_z + lz);
    }
    p.req.j_xy = nullptr;
    p.req.j_z = nullptr;
    const std::string invalid = validate(p);
    std::lock_guard<std::mutex> lock(s->mu);
    p.submit_s = now_s(s->t0);
    s->stats.submitted++;
    if (!invalid.empty()) {
        /* never queued: the request's result carries the reason */
        s->results.push_back(make_result(p, SLSF_ERR_INVALID, invalid, p.submit_s));
        s->stats.failed++;
        return SLSF_OK;
    }
    s->queue.push_back(std::move(p));
    s->cv.notify_all();
    return SLSF_OK;
}

int slsf_server_cancel(slsf_server* s, uint64_t tag) {
    if (!s) return fail(SLSF_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
        if (it->req.tag == tag) {
            slsf_result r = make_result(*it, SLSF_ERR_STATE, "cancelled", now_s(s->t0));
            s->results.push_back(r);
            s->stats.cancelled++;
            s->queue.erase(it);
            if (s->queue.empty() && s->active.empty()) s->idle.notify_all();
            return SLSF_OK;
        }
    }
    for (const Active& a : s->active)
        if (a.p.req.tag == tag) {
            s->cancel.insert(tag);
            return SLSF_OK;
        }
    /* being admitted: cancelled at the next retire */
    if (std::find(s->admitting_tags.begin(), s->admitting_tags.end(), tag) != s->admitting_tags.end()) {
        s->cancel.insert(tag);
        return SLSF_OK;
    }
    return fail(SLSF_ERR_INVALID, "unknown request tag");
}

int slsf_server_step(slsf_server* s, uint32_t* active, uint32_t* pending) {
    if (!s) return fail(SLSF_ERR_INVALID, "NULL argument");
    if (s->running) return fail(SLSF_ERR_STATE, "the server's worker thread is running");
    int rc = epoch(s);
    std::lock_guard<std::mutex> lock(s->mu);
    if (active) *active = (uint32_t)s->active.size();
    if (pending) *pending = (uint32_t)s->queue.size();
    return rc;
}

int slsf_server_start(slsf_server* s) {
    if (!s) return fail(SLSF_ERR_INVALID, "NULL argument");
    if (s->running) return SLSF_OK;
    s->stop = false;
    s->running = true;
    s->worker = std::thread([s]() {
        while (!s->stop) {
            {
                std::unique_lock<std::mutex> lock(s->mu);
                if (s->queue.empty() && s->active.empty() && s->cancel.empty())
                    s->cv.wait_for(lock, std::chrono::milliseconds(50));
            }
            if (s->stop) break;
            if (epoch(s) != SLSF_OK) {
                /* a device error ends the worker; wait_idle reports it */
                std::lock_guard<std::mutex> lock(s->mu);
                s->worker_error = g_host_error.empty() ? "device error" : g_host_error;
                s->idle.notify_all();
                break;
            }
        }
    });
    return SLSF_OK;
}

int slsf_server_wait_idle(slsf_server* s, double timeout_s) {
    if (!s) return fail(SLSF_ERR_INVALID, "NULL argument");
    std::unique_lock<std::mutex> lock(s->mu);
    const bool ok = s->idle.wait_for(lock, std::chrono::duration<double>(timeout_s), [&] {
        return (s->queue.empty() && s->active.empty() && !s->admitting) || !s->worker_error.empty();
    });
    if (!s->worker_error.empty()) return fail(SLSF_ERR_CUDA, "server worker stopped: " + s->worker_error);
    return ok ? SLSF_OK : fail(SLSF_ERR_TIMEOUT, "server still has queued or running requests");
}

int slsf_server_take_bins(slsf_server* s, uint64_t tag, double* out, size_t max_rows, size_t* n_rows) {
    if (!s || !n_rows) return fail(SLSF_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->kept_bins.find(tag);
    if (it == s->kept_bins.end()) return fail(SLSF_ERR_INVALID, "no bins kept for this tag");
    const size_t rows = it->second.size() / SLSF_BIN_COLS;
    *n_rows = rows;
    if (out && max_rows >= rows) {
        std::copy(it->second.begin(), it->second.end(), out);
        s->kept_bins.erase(it);
    }
    return SLSF_OK;
}

int slsf_server_poll(slsf_server* s, slsf_result* out, size_t max, size_t* n) {
    if (!s || (!out && max)) return fail(SLSF_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    const size_t k = std::min(max, s->results.size());
    for (size_t i = 0; i < k; ++i) out[i] = s->results[i];
    s->results.erase(s->results.begin(), s->results.begin() + k);
    if (n) *n = k;
    return SLSF_OK;
}

int slsf_server_stats_get(slsf_server* s, slsf_server_stats* out) {
    if (!s || !out) return fail(SLSF_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->stats;
    return SLSF_OK;
}

/* ---- checkpoints ----
 * One file per unfinished request, request_<tag>.ckpt: RequestRecord, J_xy
 * and J_z (FP64, L_z each), then, for a running request, the task's device
 * state (slsf_task_state_save). */
namespace {

struct RequestRecord {
    char magic[8]; /* "SLSFRQ01" */
    uint64_t tag, seed;
    uint32_t lx, ly, lz, wolff_steps;
    double temperature, proposal_width;
    uint32_t sweeps, thermalization, n_bins, binsize;
    uint32_t running, remaining, plan_binsize, plan_n_bins;
    uint64_t accepted, cluster_sites, state_bytes;
};
constexpr char kRequestMagic[8] = {'S', 'L', 'S', 'F', 'R', 'Q', '0', '1'};

int write_request(const std::string& dir, const Pending& p, const Active* a) {
    RequestRecord r;
    std::memset(&r, 0, sizeof(r));
    std::memcpy(r.magic, kRequestMagic, 8);
    r.tag = p.req.tag, r.seed = p.req.seed;
    r.lx = p.req.lx, r.ly = p.req.ly, r.lz = p.req.lz, r.wolff_steps = p.req.wolff_steps;
    r.temperature = p.req.temperature, r.proposal_width = p.req.proposal_width;
    r.sweeps = p.req.sweeps, r.thermalization = p.req.thermalization, r.n_bins = p.req.n_bins;
    r.binsize = p.req.binsize;
    std::vector<char> state;
    if (a) {
        size_t n = 0;
        if (int rc = slsf_task_state_size(a->task, &n)) return gpu_fail(rc);
        state.resize(n);
        if (int rc = slsf_task_state_save(a->task, nullptr, state.data(), n)) return gpu_fail(rc);
        r.running = 1, r.remaining = a->remaining, r.plan_binsize = a->binsize, r.plan_n_bins = a->n_bins;
        r.accepted = a->accepted, r.cluster_sites = a->cluster_sites, r.state_bytes = n;
    }
    const std::string path = dir + "/request_" + std::to_string(p.req.tag) + ".ckpt";
    const std::string tmp = path + ".tmp";
    std::FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return fail(SLSF_ERR_INVALID, "cannot write " + tmp);
    bool ok = std::fwrite(&r, sizeof(r), 1, f) == 1;
    ok = ok && std::fwrite(p.jxy.data(), 8, p.jxy.size(), f) == p.jxy.size();
    ok = ok && std::fwrite(p.jz.data(), 8, p.jz.size(), f) == p.jz.size();
    ok = ok && (state.empty() || std::fwrite(state.data(), 1, state.size(), f) == state.size());
    ok = (std::fclose(f) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) return fail(SLSF_ERR_INVALID, "cannot write " + path);
    return SLSF_OK;
}

int read_request(const std::string& path, Pending* p) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return fail(SLSF_ERR_INVALID, "cannot read " + path);
    RequestRecord r;
    bool ok = std::fread(&r, sizeof(r), 1, f) == 1 && std::memcmp(r.magic, kRequestMagic, 8) == 0;
    if (ok) {
        std::memset(&p->req, 0, sizeof(p->req));
        p->req.tag = r.tag, p->req.seed = r.seed;
        p->req.lx = r.lx, p->req.ly = r.ly, p->req.lz = r.lz, p->req.wolff_steps = r.wolff_steps;
        p->req.temperature = r.temperature, p->req.proposal_width = r.proposal_width;
        p->req.sweeps = r.sweeps, p->req.thermalization = r.thermalization, p->req.n_bins = r.n_bins;
        p->req.binsize = r.binsize;
        p->jxy.resize(r.lz);
        p->jz.resize(r.lz);
        ok = std::fread(p->jxy.data(), 8, r.lz, f) == r.lz && std::fread(p->jz.data(), 8, r.lz, f) == r.lz;
    }
    if (ok && r.running) {
        p->state.resize(r.state_bytes);
        ok = r.state_bytes > 0 && std::fread(p->state.data(), 1, r.state_bytes, f) == r.state_bytes &&
             r.plan_binsize > 0 && r.plan_n_bins > 0 && r.remaining <= r.sweeps;
        p->plan_binsize = r.plan_binsize, p->plan_n_bins = r.plan_n_bins, p->remaining = r.remaining;
        p->accepted = r.accepted, p->cluster_sites = r.cluster_sites;
    }
    ok = ok && std::fgetc(f) == EOF;
    std::fclose(f);
    if (!ok) return fail(SLSF_ERR_INVALID, "not a request checkpoint: " + path);
    return SLSF_OK;
}

}  // namespace

int slsf_server_checkpoint(slsf_server* s, const char* dir, size_t* n_saved) {
    if (!s || !dir) return fail(SLSF_ERR_INVALID, "NULL argument");
    if (s->running) return fail(SLSF_ERR_STATE, "the server's worker thread is running; stop it first");
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) return fail(SLSF_ERR_INVALID, std::string("cannot create ") + dir);
    std::lock_guard<std::mutex> lock(s->mu);
    size_t n = 0;
    for (const Active& a : s->active) {
        if (s->cancel.count(a.p.req.tag)) continue;
        if (int rc = write_request(dir, a.p, &a)) return rc;
        ++n;
    }
    for (const Pending& p : s->queue) {
        if (int rc = write_request(dir, p, nullptr)) return rc;
        ++n;
    }
    if (n_saved) *n_saved = n;
    return SLSF_OK;
}

int slsf_server_restore(slsf_server* s, const char* dir, size_t* n_restored) {
    if (!s || !dir) return fail(SLSF_ERR_INVALID, "NULL argument");
    std::vector<Pending> got;
    std::error_code ec;
    for (const auto& e : std::filesystem::directory_iterator(dir, ec)) {
        const std::string name = e.path().filename().string();
        if (name.rfind("request_", 0) != 0 || e.path().extension() != ".ckpt") continue;
        Pending p;
        if (int rc = read_request(e.path().string(), &p)) return rc;
        got.push_back(std::move(p));
    }
    if (ec) return fail(SLSF_ERR_INVALID, std::string("cannot read ") + dir);
    std::sort(got.begin(), got.end(), [](const Pending& a, const Pending& b) { return a.req.tag < b.req.tag; });
    std::lock_guard<std::mutex> lock(s->mu);
    for (Pending& p : got) {
        p.submit_s = now_s(s->t0);
        s->stats.submitted++;
        const std::string invalid = validate(p);
        if (!invalid.empty()) {
            s->results.push_back(make_result(p, SLSF_ERR_INVALID, invalid, p.submit_s));
            s->stats.failed++;
            continue;
        }
        s->queue.push_back(std::move(p));
    }
    s->cv.notify_all();
    if (n_restored) *n_restored = got.size();
    return SLSF_OK;
}

}  // extern "C"
