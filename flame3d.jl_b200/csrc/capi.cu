// capi.cu — error reporting and argument checks shared by every C entry point.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "common.cuh"

namespace {
thread_local char g_err[512] = "";
}

int flame_fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

// Launch errors (bad configuration, missing sm_100a image) surface here.  Errors of earlier
// asynchronous work that are sticky are reported too, so the caller never continues on a
// broken context without being told.
int flame_check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return flame_fail(FLAME_ELAUNCH, "%s: %s (%s)", what, cudaGetErrorName(e),
                          cudaGetErrorString(e));
    return FLAME_OK;
}

int flame_check_grid(const FlameGrid *g, const char *what) {
    if (!g) return flame_fail(FLAME_EINVAL, "%s: grid is NULL", what);
    if (g->ng != FLAME_NG)
        return flame_fail(FLAME_EINVAL, "%s: ng=%d, the stencils need ng=%d", what, g->ng,
                          FLAME_NG);
    if (g->nx < 1 || g->ny < 1 || g->nz < 1)
        return flame_fail(FLAME_EINVAL, "%s: interior extents %dx%dx%d must be positive", what,
                          g->nx, g->ny, g->nz);
    if (g->ns < 1 || g->ns > FLAME_MAX_NS)
        return flame_fail(FLAME_EINVAL, "%s: ns=%d outside 1..%d", what, g->ns, FLAME_MAX_NS);
    return FLAME_OK;
}

extern "C" {

int flame_last_error(char *buf, size_t n) {
    size_t len = strlen(g_err);
    if (buf && n) {
        size_t c = len < n - 1 ? len : n - 1;
        memcpy(buf, g_err, c);
        buf[c] = 0;
    }
    return (int)len;
}

int flame_version(void) { return 10000; }

}  // extern "C"
