// C ABI of libincrmt_gpu (declared in include/incrmt.h): multigrid solver
// handles and the thread-local error message.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include "common.cuh"
#include "mg.cuh"


namespace incrmt {

thread_local char g_last_error[512] = {0};

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

int cuda_status(cudaError_t e, const char *what, const char *file, int line) {
    set_error("%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    return e == cudaErrorMemoryAllocation ? INCRMT_ERR_OOM : INCRMT_ERR_CUDA;
}

}  // namespace incrmt

using incrmt::set_error;

extern "C" {

const char *incrmt_last_error(void) { return incrmt::g_last_error; }

int incrmt_mg_create(int sys, int m, int n, double ax, double bx, double ay, double by,
                     int x_prd, int y_prd, int zpr, incrmt_mg **out) {
    if (!out) { set_error("null output pointer"); return INCRMT_ERR_BADARG; }
    *out = nullptr;
    incrmt_mg *h = new (std::nothrow) incrmt_mg;
    if (!h) { set_error("host allocation failed"); return INCRMT_ERR_OOM; }
    int r = h->mg.create(sys, m, n, ax, bx, ay, by, x_prd, y_prd, zpr);
    if (r != INCRMT_OK) { h->mg.destroy(); delete h; return r; }
    *out = h;
    return INCRMT_OK;
}

int incrmt_mg_size(const incrmt_mg *h, int *m_sys, int *n_sys) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    if (m_sys) *m_sys = h->mg.m;
    if (n_sys) *n_sys = h->mg.n;
    return INCRMT_OK;
}

int incrmt_mg_set_density_device(incrmt_mg *h, const double *d_rho) {
    if (!h || !d_rho) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Multigrid &g = h->mg;
    if (g.coarse_every <= 1) return g.set_density_device(d_rho);
    // Lagged coarse levels may be rebuilt at the next solve: keep the
    // density in the handle's own buffer until then.
    const size_t bytes = sizeof(double) * (g.cm + 4) * (g.cn + 4);
    INCRMT_CK(cudaMemcpyAsync(g.rho, d_rho, bytes, cudaMemcpyDeviceToDevice, g.stream));
    return g.set_density_lagged(g.rho, 0);
}

int incrmt_mg_set_density(incrmt_mg *h, const double *rho) {
    if (!h || !rho) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Multigrid &g = h->mg;
    const size_t bytes = sizeof(double) * (g.cm + 4) * (g.cn + 4);
    INCRMT_CK(cudaMemcpyAsync(g.rho, rho, bytes, cudaMemcpyHostToDevice, g.stream));
    int r = g.set_density_lagged(g.rho, 0);
    if (r != INCRMT_OK) return r;
    INCRMT_CK(cudaStreamSynchronize(g.stream));
    return INCRMT_OK;
}

int incrmt_mg_solve_device(incrmt_mg *h, const double *d_b, double *d_z,
                           const incrmt_mg_opts *opts, incrmt_mg_stats *stats) {
    if (!h || !d_b || !d_z) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    return h->mg.solve_lagged(d_b, d_z, opts, stats, true);
}

int incrmt_mg_solve(incrmt_mg *h, const double *b, double *z,
                    const incrmt_mg_opts *opts, incrmt_mg_stats *stats) {
    if (!h || !b || !z) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Multigrid &g = h->mg;
    const size_t bytes = sizeof(double) * g.m * g.n;
    INCRMT_CK(cudaMemcpyAsync(g.bbuf, b, bytes, cudaMemcpyHostToDevice, g.stream));
    INCRMT_CK(cudaMemcpyAsync(g.zbuf, z, bytes, cudaMemcpyHostToDevice, g.stream));
    int r = g.solve_lagged(g.bbuf, g.zbuf, opts, stats, true);
    if (r != INCRMT_OK && r != INCRMT_ERR_NOCONV) return r;
    cudaError_t e1 = cudaMemcpyAsync(z, g.zbuf, bytes, cudaMemcpyDeviceToHost, g.stream);
    cudaError_t e2 = cudaStreamSynchronize(g.stream);
    if (e1 != cudaSuccess) return incrmt::cuda_status(e1, "copy solution", __FILE__, __LINE__);
    if (e2 != cudaSuccess) return incrmt::cuda_status(e2, "sync", __FILE__, __LINE__);
    return r;
}

int incrmt_mg_apply(incrmt_mg *h, const double *z, double *out) {
    if (!h || !z || !out) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    incrmt::Multigrid &g = h->mg;
    const size_t bytes = sizeof(double) * g.m * g.n;
    INCRMT_CK(cudaMemcpyAsync(g.zbuf, z, bytes, cudaMemcpyHostToDevice, g.stream));
    int r = g.apply_device(g.zbuf, g.bbuf);
    if (r != INCRMT_OK) return r;
    INCRMT_CK(cudaMemcpyAsync(out, g.bbuf, bytes, cudaMemcpyDeviceToHost, g.stream));
    INCRMT_CK(cudaStreamSynchronize(g.stream));
    return INCRMT_OK;
}

int incrmt_mg_vcycle_device(incrmt_mg *h, const double *d_b, double *d_z) {
    if (!h || !d_b || !d_z) { set_error("null argument"); return INCRMT_ERR_BADARG; }
    return h->mg.vcycle64(d_b, d_z);
}

int incrmt_mg_set_tiles(incrmt_mg *h, int on) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    incrmt::Multigrid &mg = h->mg;
    if (mg.stream) INCRMT_CK(cudaStreamSynchronize(mg.stream));
    mg.tiles = on != 0;
    if (mg.gexec) {  // the captured V-cycle holds the other launches
        cudaGraphExecDestroy(mg.gexec);
        mg.gexec = nullptr;
    }
    if (mg.setup_exec) {  // and so does the captured rebuild
        cudaGraphExecDestroy(mg.setup_exec);
        mg.setup_exec = nullptr;
    }
    if (mg.kexec) {  // and the captured Krylov iteration
        cudaGraphExecDestroy(mg.kexec);
        mg.kexec = nullptr;
    }
    return INCRMT_OK;
}

int incrmt_mg_set_krylov(incrmt_mg *h, int on) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    h->mg.krylov = on != 0;
    return INCRMT_OK;
}

long long incrmt_mg_krylov_fallbacks(const incrmt_mg *h) { return h ? h->mg.krylov_fallbacks : 0; }

int incrmt_mg_set_coarse_refresh(incrmt_mg *h, int every) {
    if (!h || every < 1) { set_error("bad argument"); return INCRMT_ERR_BADARG; }
    h->mg.coarse_every = every;
    h->mg.coarse_stale = true;
    return INCRMT_OK;
}

long long incrmt_mg_coarse_builds(const incrmt_mg *h, long long *retries) {
    if (!h) return 0;
    if (retries) *retries = h->mg.coarse_retries;
    return h->mg.coarse_builds;
}

long long incrmt_mg_mixed_fallbacks(const incrmt_mg *h) { return h ? h->mg.mixed_fallbacks : 0; }

int incrmt_mg_set_profiling(incrmt_mg *h, int on) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    h->mg.prof = on != 0;
    h->mg.prof_ms = 0; h->mg.prof_bytes = 0; h->mg.prof_launches = 0;
    return INCRMT_OK;
}

int incrmt_mg_profile(incrmt_mg *h, double *ms, double *bytes, long long *launches) {
    if (!h) { set_error("null handle"); return INCRMT_ERR_BADARG; }
    int r = h->mg.prof_collect();
    if (r) return r;
    if (ms) *ms = h->mg.prof_ms;
    if (bytes) *bytes = h->mg.prof_bytes;
    if (launches) *launches = h->mg.prof_launches;
    return INCRMT_OK;
}

void *incrmt_mg_stream(const incrmt_mg *h) { return h ? static_cast<void *>(h->mg.stream) : nullptr; }

int incrmt_mg_levels(const incrmt_mg *h) { return h ? static_cast<int>(h->mg.lev.size()) : 0; }

long long incrmt_mg_launches(const incrmt_mg *h) { return h ? h->mg.launches : 0; }

void incrmt_mg_destroy(incrmt_mg *h) {
    if (!h) return;
    if (h->mg.stream) cudaStreamSynchronize(h->mg.stream);
    h->learned.release();
    h->mg.destroy();
    delete h;
}

}  // extern "C"
