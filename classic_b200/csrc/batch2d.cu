// Host side of the batched 2D step (claw_batch_* in include/claw_b200.h):
// many independent grids of one solver and method, each with its own claw2
// dt control, advanced by one persistent launch per step over a work list of
// the rows of every instance still running; the launches are captured in
// CUDA-graph chunks and the host polls one counter per chunk.  Built with
// --fmad=false like the single-grid reference-order path.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/claw_b200.h"
#include "host.h"
#include "riemann.cuh"
#include "step2d.cuh"
#include "batch2d_runner.cuh"

using namespace clawb200;

namespace {

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

template <class S>
std::unique_ptr<BatchRunner> batch_runner(const claw_config& cfg, const S& s) {
    bool mc = cfg.order == 2 && cfg.transverse_waves == 2 && cfg.capa_index == 0 && !cfg.use_fwaves;
    for (int k = 0; k < cfg.num_waves; ++k) mc = mc && cfg.limiter[k] == 4;
    if (mc) return std::unique_ptr<BatchRunner>(new BatchRunnerT<S, MethodMC2D>(s));
    return std::unique_ptr<BatchRunner>(new BatchRunnerT<S, MethodGeneric2D>(s));
}

std::unique_ptr<BatchRunner> make_batch_runner(const claw_config& cfg) {
    if (cfg.solver_id == CLAW_SOLVER_EULER_ROE_2D) {
        const double gamma = cfg.solver_params[0];
        return batch_runner(cfg, EulerRoe2D<double>{gamma, gamma - 1.0});
    }
    if (cfg.solver_id == CLAW_SOLVER_ACOUSTICS_2D) {
        const double rho = cfg.solver_params[0], bulk = cfg.solver_params[1];
        const double cc = std::sqrt(bulk / rho), zz = rho * cc, hz = 0.5 / zz;
        return batch_runner(cfg, Acoustics2D<double>{cc, zz, hz});
    }
    return nullptr;
}

// every field but the grid size must agree with instance 0
bool same_method(const claw_config& a, const claw_config& b) {
    if (a.num_dim != b.num_dim || a.num_eqn != b.num_eqn || a.num_waves != b.num_waves ||
        a.num_aux != b.num_aux || a.capa_index != b.capa_index || a.order != b.order ||
        a.transverse_waves != b.transverse_waves || a.use_fwaves != b.use_fwaves ||
        a.solver_id != b.solver_id || a.precision != b.precision || a.num_ghost != b.num_ghost)
        return false;
    for (int k = 0; k < CLAW_MAX_WAVES; ++k)
        if (a.limiter[k] != b.limiter[k]) return false;
    for (int d = 0; d < 2; ++d)
        if (a.bc_lower[d] != b.bc_lower[d] || a.bc_upper[d] != b.bc_upper[d]) return false;
    for (int k = 0; k < 8; ++k)
        if (a.solver_params[k] != b.solver_params[k]) return false;
    return true;
}

}  // namespace

struct claw_batch {
    std::vector<claw_config> cfgs;
    std::vector<Geometry> g;
    cudaStream_t stream = nullptr;
    ClawCtl* ctl_d = nullptr;
    ClawCtl* ctl_h = nullptr;  // pinned
    int* flags_d = nullptr;    // [0] active instances, [1] error flags
    int* flags_h = nullptr;    // pinned
    std::unique_ptr<BatchRunner> runner;
    cudaGraphExec_t gexec = nullptr;
    int gsteps = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long launches = 0;
    int device = 0;

    // Frees everything the batch holds, so an error part-way through
    // claw_batch_create leaks nothing.
    ~claw_batch() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        if (gexec) cudaGraphExecDestroy(gexec);
        runner.reset();
        for (auto& gg : g) {
            for (int s = 0; s < 2; ++s)
                if (gg.q[s]) cudaFree(gg.q[s]);
            if (gg.aux) cudaFree(gg.aux);
        }
        if (ctl_d) cudaFree(ctl_d);
        if (ctl_h) cudaFreeHost(ctl_h);
        if (flags_d) cudaFree(flags_d);
        if (flags_h) cudaFreeHost(flags_h);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

int claw_batch_create(const claw_config* cfgs, int count, claw_batch** out) {
    if (!out || !cfgs) return fail(CLAW_E_INVALID, "null argument");
    *out = nullptr;
    if (count < 1 || count > BATCH_MAX) return fail(CLAW_E_INVALID, "batch size must be 1..%d", BATCH_MAX);
    for (int k = 0; k < count; ++k) {
        if (cfgs[k].num_dim != 2) return fail(CLAW_E_UNSUPPORTED, "batches are 2D");
        if (!same_method(cfgs[0], cfgs[k]))
            return fail(CLAW_E_INVALID, "instance %d differs from instance 0 in more than its grid", k);
        if (cfgs[k].precision != CLAW_FP64 && cfgs[k].precision != CLAW_FP64_FMA)
            return fail(CLAW_E_UNSUPPORTED, "batches run in FP64 (CLAW_FP64 or CLAW_FP64_FMA)");
        if (cfgs[k].num_ghost != 2) return fail(CLAW_E_INVALID, "num_ghost must be 2");
        if (cfgs[k].dimensional_split != 0 || cfgs[k].source_split != 0)
            return fail(CLAW_E_UNSUPPORTED, "splitting / source terms are not built");
        for (int d = 0; d < 2; ++d) {
            if (cfgs[k].num_cells[d] < 2) return fail(CLAW_E_INVALID, "num_cells[%d] must be >= 2", d);
            if (!(cfgs[k].upper[d] > cfgs[k].lower[d])) return fail(CLAW_E_INVALID, "upper <= lower");
            for (int side = 0; side < 2; ++side) {
                const int bc = side ? cfgs[k].bc_upper[d] : cfgs[k].bc_lower[d];
                if (bc < 1 || bc > 3) return fail(CLAW_E_UNSUPPORTED, "boundary condition %d", bc);
            }
        }
    }
    std::unique_ptr<claw_batch> b(new claw_batch());
    b->cfgs.assign(cfgs, cfgs + count);
    b->runner = cfgs[0].precision == CLAW_FP64_FMA ? make_fast_batch_runner(cfgs[0])
                                                   : make_batch_runner(cfgs[0]);
    if (!b->runner) return fail(CLAW_E_UNSUPPORTED, "no batch kernel for solver %d", cfgs[0].solver_id);
    CUDA_TRY(cudaGetDevice(&b->device));
    CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreate(&b->ev0));
    CUDA_TRY(cudaEventCreate(&b->ev1));
    CUDA_TRY(cudaMalloc(&b->ctl_d, sizeof(ClawCtl) * count));
    CUDA_TRY(cudaMallocHost(&b->ctl_h, sizeof(ClawCtl) * count));
    std::memset(b->ctl_h, 0, sizeof(ClawCtl) * count);
    for (int k = 0; k < count; ++k) b->ctl_h[k].done = 1;
    CUDA_TRY(cudaMemcpy(b->ctl_d, b->ctl_h, sizeof(ClawCtl) * count, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMalloc(&b->flags_d, 2 * sizeof(int)));
    CUDA_TRY(cudaMallocHost(&b->flags_h, 2 * sizeof(int)));
    CUDA_TRY(cudaMemset(b->flags_d, 0, 2 * sizeof(int)));
    b->g.resize(count);
    for (int k = 0; k < count; ++k) {
        Geometry& g = b->g[k];
        std::memset(&g, 0, sizeof(g));
        const claw_config& c = cfgs[k];
        g.dim = 2;
        g.mx = c.num_cells[0];
        g.my = c.num_cells[1];
        g.mz = 1;
        g.meqn = c.num_eqn;
        g.maux = c.num_aux;
        g.es = 8;
        g.dx = (c.upper[0] - c.lower[0]) / (double)(float)g.mx;
        g.dy = (c.upper[1] - c.lower[1]) / (double)(float)g.my;
        g.dz = 1.0;
        g.ld = round_up(g.mx, 32);
        g.fstride = g.ld * g.my;
        g.ald = round_up(g.mx + 4, 4);
        g.afstride = g.ald * (g.my + 4);
        const size_t qbytes = (size_t)g.fstride * g.meqn * 8;
        for (int s = 0; s < 2; ++s) {
            CUDA_TRY(cudaMalloc(&g.q[s], qbytes));
            CUDA_TRY(cudaMemsetAsync(g.q[s], 0, qbytes, b->stream));
        }
        if (g.maux > 0) {
            const size_t abytes = (size_t)g.afstride * g.maux * 8;
            CUDA_TRY(cudaMalloc(&g.aux, abytes));
            CUDA_TRY(cudaMemsetAsync(g.aux, 0, abytes, b->stream));
        }
        g.ctl = b->ctl_d + k;
    }
    int rc = b->runner->prepare(b->g, cfgs, b->ctl_d, b->flags_d, b->flags_d + 1);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    *out = b.release();
    return 0;
}

int claw_batch_destroy(claw_batch* b) {
    delete b;  // ~claw_batch frees the device state
    return 0;
}

static int batch_fields(claw_batch* b, int k, double* host, bool to_device) {
    const Geometry& g = b->g[k];
    const int cur = b->ctl_h[k].cur;
    for (int m = 0; m < g.meqn; ++m) {
        char* d = static_cast<char*>(g.q[cur]) + (size_t)m * g.fstride * 8;
        double* hp = host + (size_t)m * g.mx * g.my;
        if (to_device)
            CUDA_TRY(cudaMemcpy2DAsync(d, g.ld * 8, hp, g.mx * 8, g.mx * 8, g.my,
                                       cudaMemcpyHostToDevice, b->stream));
        else
            CUDA_TRY(cudaMemcpy2DAsync(hp, g.mx * 8, d, g.ld * 8, g.mx * 8, g.my,
                                       cudaMemcpyDeviceToHost, b->stream));
    }
    return 0;
}

int claw_batch_set_q(claw_batch* b, int k, const double* q) {
    if (!b || !q || k < 0 || k >= (int)b->g.size()) return fail(CLAW_E_INVALID, "bad argument");
    CUDA_TRY(cudaSetDevice(b->device));
    int rc = batch_fields(b, k, const_cast<double*>(q), true);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return 0;
}

int claw_batch_get_q(claw_batch* b, int k, double* q) {
    if (!b || !q || k < 0 || k >= (int)b->g.size()) return fail(CLAW_E_INVALID, "bad argument");
    CUDA_TRY(cudaSetDevice(b->device));
    int rc = batch_fields(b, k, q, false);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return 0;
}

static int batch_graph(claw_batch* b, int steps) {
    if (b->gexec && b->gsteps == steps) return 0;
    if (b->gexec) {
        cudaGraphExecDestroy(b->gexec);
        b->gexec = nullptr;
    }
    cudaGraph_t graph;
    CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < steps; ++s) {
        cudaError_t e = b->runner->launch(b->stream);
        if (e != cudaSuccess) {
            cudaStreamEndCapture(b->stream, &graph);
            return fail(CLAW_E_CUDA, "launch during capture: %s", cudaGetErrorString(e));
        }
    }
    CUDA_TRY(cudaStreamEndCapture(b->stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&b->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(CLAW_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    b->gsteps = steps;
    return 0;
}

int claw_batch_advance(claw_batch* b, double tstart, double tend, const double* dt_initial,
                       claw_stats* stats) {
    if (!b) return fail(CLAW_E_INVALID, "null batch");
    CUDA_TRY(cudaSetDevice(b->device));
    const int n = (int)b->g.size();
    std::vector<int> info(n, 0);
    int active = 0;
    for (int k = 0; k < n; ++k) {
        const claw_config& cfg = b->cfgs[k];
        ClawCtl* c = &b->ctl_h[k];
        const int cur = c->cur;
        std::memset(c, 0, sizeof(ClawCtl));
        const double dt0 = dt_initial ? dt_initial[k] : cfg.dt_initial;
        c->cur = cur;
        c->t = c->told = tstart;
        c->tstart = tstart;
        c->tend = tend;
        c->dt = dt0;
        c->dt_max = cfg.dt_max;
        c->cfl_max = cfg.cfl_max;
        c->cfl_desired = cfg.cfl_desired;
        c->dtmin = c->dtmax = dt0;
        c->mode = CTL_ADVANCE;
        c->dt_variable = cfg.dt_variable ? 1 : 0;
        int maxn = cfg.steps_max;
        // claw2's argument checks, per instance (src/2d/claw2.f:508-543)
        if (!cfg.dt_variable) {
            if (tend < tstart) maxn = 1;
            else {
                maxn = (int)std::lround((tend - tstart) / dt0);
                if (std::fabs(maxn * dt0 - (tend - tstart)) > 1e-5 * (tend - tstart)) info[k] = 2;
            }
        }
        if (!info[k] && cfg.dt_variable && cfg.cfl_desired > cfg.cfl_max) info[k] = 3;
        if (!info[k] && cfg.capa_index > cfg.num_aux) info[k] = 5;
        if (!info[k] && cfg.order < cfg.transverse_waves) info[k] = 6;
        c->maxn = maxn;
        c->done = (info[k] != 0 || maxn == 0) ? 1 : 0;
        if (!c->done && c->told + c->dt > tend && tstart < tend) c->dt = tend - c->told;
        active += c->done ? 0 : 1;
    }
    CUDA_TRY(cudaMemcpyAsync(b->ctl_d, b->ctl_h, sizeof(ClawCtl) * n, cudaMemcpyHostToDevice, b->stream));
    b->flags_h[0] = active;
    b->flags_h[1] = 0;
    CUDA_TRY(cudaMemcpyAsync(b->flags_d, b->flags_h, 2 * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    const long long launches0 = b->launches;
    CUDA_TRY(cudaEventRecord(b->ev0, b->stream));
    if (active > 0) {
        const int chunk = 16;
        int rc = batch_graph(b, chunk);
        if (rc) return rc;
        for (;;) {
            CUDA_TRY(cudaGraphLaunch(b->gexec, b->stream));
            b->launches += chunk;
            CUDA_TRY(cudaMemcpyAsync(b->flags_h, b->flags_d, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                                     b->stream));
            CUDA_TRY(cudaStreamSynchronize(b->stream));
            if (b->flags_h[1] != 0 || b->flags_h[0] <= 0) break;
        }
    }
    CUDA_TRY(cudaEventRecord(b->ev1, b->stream));
    CUDA_TRY(cudaMemcpyAsync(b->ctl_h, b->ctl_d, sizeof(ClawCtl) * n, cudaMemcpyDeviceToHost, b->stream));
    CUDA_TRY(cudaEventSynchronize(b->ev1));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    int first = 0;
    for (int k = 0; k < n; ++k) {
        const claw_config& cfg = b->cfgs[k];
        const ClawCtl* c = &b->ctl_h[k];
        if (!info[k] && cfg.dt_variable && c->t < tend && c->n == c->maxn) info[k] = 11;
        if (!info[k] && !cfg.dt_variable && c->cflmax_seen > cfg.cfl_max) info[k] = 12;
        if ((c->err | b->flags_h[1]) & CTL_ERR_TMA_TIMEOUT) info[k] = CLAW_E_DEVICE;
        else if (c->err & CTL_ERR_NAN_CFL) info[k] = CLAW_E_NAN;
        if (stats) {
            claw_stats* st = &stats[k];
            st->t_reached = c->t;
            st->dt_min = c->dtmin;
            st->dt_max_taken = c->dtmax;
            st->dt_next = c->dt;
            st->cfl_max_seen = c->cflmax_seen;
            st->cfl_last = c->cfl_last;
            st->steps_taken = c->n;
            st->steps_rejected = c->nrej;
            st->info = info[k];
            st->device_error = c->err;
            st->device_ms = ms;
            st->launches = b->launches - launches0;
        }
        if (!first && info[k]) first = info[k];
    }
    if (first < 0) return fail(first, "device error in the batch");
    return first;
}

int claw_batch_autotune(claw_batch* b, const double* dt_trial, int repeats, int* min_rows,
                        int* ctas_per_sm, double* ms_per_step) {
    if (!b) return fail(CLAW_E_INVALID, "null batch");
    if (repeats < 1) repeats = 1;
    CUDA_TRY(cudaSetDevice(b->device));
    const int n = (int)b->g.size();
    // trial steps start every instance afresh from its current q: the kernel
    // reads q[cur] and writes q[cur ^ 1], and the saved control blocks are
    // put back before every trial and at the end, so the state is unchanged
    std::vector<ClawCtl> saved(b->ctl_h, b->ctl_h + n), trial(n);
    for (int k = 0; k < n; ++k) {
        const claw_config& cfg = b->cfgs[k];
        ClawCtl& c = trial[k];
        std::memset(&c, 0, sizeof(ClawCtl));
        c.cur = saved[k].cur;
        c.tend = 1e300;
        c.dt = dt_trial ? dt_trial[k] : cfg.dt_initial;
        c.dt_max = cfg.dt_max;
        c.cfl_max = cfg.cfl_max;
        c.cfl_desired = cfg.cfl_desired;
        c.dtmin = c.dtmax = c.dt;
        c.mode = CTL_ADVANCE;
        c.dt_variable = cfg.dt_variable ? 1 : 0;
        c.maxn = 1;
    }
    // Two regimes: while many instances run, the launch is full whatever the
    // tile height and the CTA count decides; once only the largest ones are
    // left (the tail of an uneven ensemble) the tile height decides how many
    // warps share them.  The CTA count is tuned on a step of every instance,
    // the tile height on a step of the largest instance alone.
    std::vector<ClawCtl> tail = trial;
    int big = 0;
    for (int k = 1; k < n; ++k)
        if ((long long)b->g[k].mx * b->g[k].my > (long long)b->g[big].mx * b->g[big].my) big = k;
    for (int k = 0; k < n; ++k) tail[k].done = k == big ? 0 : 1;
    auto time_step = [&](const std::vector<ClawCtl>& st, int active, float* out) -> int {
        float tmin = 1e30f;
        for (int r = 0; r < repeats; ++r) {
            std::memcpy(b->ctl_h, st.data(), sizeof(ClawCtl) * n);
            CUDA_TRY(cudaMemcpyAsync(b->ctl_d, b->ctl_h, sizeof(ClawCtl) * n, cudaMemcpyHostToDevice,
                                     b->stream));
            b->flags_h[0] = active;
            b->flags_h[1] = 0;
            CUDA_TRY(cudaMemcpyAsync(b->flags_d, b->flags_h, 2 * sizeof(int), cudaMemcpyHostToDevice,
                                     b->stream));
            CUDA_TRY(cudaEventRecord(b->ev0, b->stream));
            CUDA_TRY(b->runner->launch(b->stream));
            CUDA_TRY(cudaEventRecord(b->ev1, b->stream));
            CUDA_TRY(cudaEventSynchronize(b->ev1));
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
            tmin = std::min(tmin, ms);
        }
        *out = tmin;
        return 0;
    };
    const int maxc = b->runner->max_ctas_per_sm();
    float best = 1e30f, best_tail = 1e30f;
    int best_ctas = maxc, best_rows = 48;
    for (int ctas = maxc; ctas >= 1 && ctas >= maxc / 2; --ctas) {
        b->runner->set_shape(48, ctas);
        float t = 0.f;
        int rc = time_step(trial, n, &t);
        if (rc) return rc;
        if (t < best) { best = t; best_ctas = ctas; }
    }
    const int rows_cand[] = {16, 24, 32, 48, 96, 192};
    for (int rows : rows_cand) {
        b->runner->set_shape(rows, best_ctas);
        float t = 0.f;
        int rc = time_step(tail, 1, &t);
        if (rc) return rc;
        if (t < best_tail) { best_tail = t; best_rows = rows; }
    }
    b->runner->set_shape(best_rows, best_ctas);
    if (b->gexec) {  // the captured time loop holds the old launch shape
        cudaGraphExecDestroy(b->gexec);
        b->gexec = nullptr;
        b->gsteps = 0;
    }
    std::memcpy(b->ctl_h, saved.data(), sizeof(ClawCtl) * n);
    CUDA_TRY(cudaMemcpyAsync(b->ctl_d, b->ctl_h, sizeof(ClawCtl) * n, cudaMemcpyHostToDevice, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (min_rows) *min_rows = best_rows;
    if (ctas_per_sm) *ctas_per_sm = best_ctas;
    if (ms_per_step) *ms_per_step = best;
    return 0;
}

int claw_batch_set_shape(claw_batch* b, int min_rows, int ctas_per_sm) {
    if (!b || min_rows < 1 || ctas_per_sm < 1) return fail(CLAW_E_INVALID, "bad argument");
    b->runner->set_shape(min_rows, ctas_per_sm);
    if (b->gexec) {
        cudaGraphExecDestroy(b->gexec);
        b->gexec = nullptr;
        b->gsteps = 0;
    }
    return 0;
}

}  // extern "C"
