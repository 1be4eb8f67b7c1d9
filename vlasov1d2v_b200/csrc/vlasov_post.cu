// Device kernels around the time loop: initial-state construction, edge smoothing and
// fine-grid interpolation of the nodal state (declarations and reference citations in
// include/vlasov1d2v.h).
//
// All three are memory-bound elementwise or small-contraction passes over the ghost-inclusive
// state f[X][n][U][n][V][n].  Products and sums are written with explicit round-to-nearest
// intrinsics (no FMA contraction) in the order the reference's NumPy/CuPy expressions
// evaluate them, so results match the reference bit for bit given the same host tables.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "vlasov1d2v.h"

void vl_internal_set_error(const char *msg);

namespace {

int fail(int code, const char *msg) {
    vl_internal_set_error(msg);
    return code;
}

int check(const char *where) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        vl_internal_set_error((std::string(where) + ": " + cudaGetErrorString(e)).c_str());
        return VL_ERR_CUDA;
    }
    return VL_OK;
}

// ---------------------------------------------------------------------------------------------
// initial state: f[e,i,a,j,b,k] = pol[a,j,b,k] * mx[e,i] + scale * (cx[e,i] vre - sx[e,i] vim)
// ---------------------------------------------------------------------------------------------
template <typename T>
__global__ void initial_state_kernel(T *__restrict__ f, const double *__restrict__ pol,
                                     const double *__restrict__ mx, const double *__restrict__ cx,
                                     const double *__restrict__ sx, const double *__restrict__ vre,
                                     const double *__restrict__ vim, double scale, int64_t vel,
                                     int64_t total) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t xi = p / vel, q = p - xi * vel;   // x node (e, i) and velocity node
        double v = pol[q];
        if (mx != nullptr) v = __dmul_rn(v, mx[xi]);
        if (vre != nullptr) {
            // real part of exp(i k x) * mode, times 2 delta_n (main/grid.py:238-240)
            const double re = __dsub_rn(__dmul_rn(cx[xi], vre[q]), __dmul_rn(sx[xi], vim[q]));
            v = __dadd_rn(v, __dmul_rn(scale, re));
        }
        f[p] = (T)v;
    }
}

// ---------------------------------------------------------------------------------------------
// smooth_edges (main/grid.py:116-134): six in-place passes, each averaging one face-node plane
// of every interior element with its neighbour's opposite face plane, in the reference's order
// (x left, x right, u left, u right, v left, v right); each pass sees the previous passes.
// ---------------------------------------------------------------------------------------------
template <typename T>
__global__ void smooth_pass_kernel(T *__restrict__ f, int axis, int side, int nx, int nu, int nv,
                                   int n) {
    const int X = nx + 2, U = nu + 2, V = nv + 2;
    const int64_t sk = 1, sb = n, sj = (int64_t)V * n, sa = sj * n, si = sa * U, se = si * n;
    // enumerate the interior face plane: the axis' node index is fixed
    const int ext[3] = {nx, nu, nv};
    const int64_t total = (int64_t)ext[0] * ext[1] * ext[2] * n * n;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total;
         p += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = p;
        // order of the free indices (outer to inner): e, a, b and the two free nodes
        int e, a, b, na, nb;   // na, nb = node indices of the two non-axis directions
        nb = (int)(r % n); r /= n;
        na = (int)(r % n); r /= n;
        b = (int)(r % nv) + 1; r /= nv;
        a = (int)(r % nu) + 1; r /= nu;
        e = (int)r + 1;
        int i, j, k;
        int64_t step;   // element stride along the axis
        int nd = side == 0 ? 0 : n - 1;          // node written
        int no = side == 0 ? n - 1 : 0;          // neighbour's node read
        int64_t base;
        if (axis == 0) {
            j = na; k = nb; step = se;
            base = e * se + a * sa + j * sj + b * sb + k * sk;
            const int64_t pw = base + nd * si;
            const int64_t pr = base + (side == 0 ? -step : step) + no * si;
            f[pw] = (T)__dmul_rn(0.5, __dadd_rn((double)f[pr], (double)f[pw]));
        } else if (axis == 1) {
            i = na; k = nb; step = sa;
            base = e * se + i * si + a * sa + b * sb + k * sk;
            const int64_t pw = base + nd * sj;
            const int64_t pr = base + (side == 0 ? -step : step) + no * sj;
            f[pw] = (T)__dmul_rn(0.5, __dadd_rn((double)f[pr], (double)f[pw]));
        } else {
            i = na; j = nb; step = sb;
            base = e * se + i * si + a * sa + j * sj + b * sb;
            const int64_t pw = base + nd * sk;
            const int64_t pr = base + (side == 0 ? -step : step) + no * sk;
            f[pw] = (T)__dmul_rn(0.5, __dadd_rn((double)f[pr], (double)f[pw]));
        }
        (void)X;
    }
}

// ---------------------------------------------------------------------------------------------
// Basis3D.interpolate_values (main/basis.py:291-317): per element (e, a, b) of the range,
//   out[p][q][r] = sum_k ell_v[b][k][r] sum_j ell_u[a][j][q] sum_i ell_x[e][i][p] f[e,i,a,j,b,k]
// contracted x first, then u, then v, each sum sequential over the node index.
// out layout: [ex][fx][eu][fu][ev][fv] over the element range.
// ---------------------------------------------------------------------------------------------
constexpr int INTERP_THREADS = 256;
constexpr int INTERP_MAX_N = 10;
constexpr int INTERP_MAX_FINE = 32;

template <typename T>
__global__ void __launch_bounds__(INTERP_THREADS)
interpolate_kernel(const T *__restrict__ f, int nu, int nv, int n, int e0, int a0, int b0,
                   int ex, int eu, int ev, const double *__restrict__ lx,
                   const double *__restrict__ lu, const double *__restrict__ lv, int fx, int fu,
                   int fv, double *__restrict__ out) {
    extern __shared__ double sm[];
    double *blk = sm;                       // [n][n][n]   f of the element (i, j, k)
    double *g1 = blk + n * n * n;           // [fx][n][n]  after x
    double *g2 = g1 + fx * n * n;           // [fx][fu][n] after u
    const int le = blockIdx.z, la = blockIdx.y, lb = blockIdx.x;   // element within the range
    const int e = e0 + le, a = a0 + la, b = b0 + lb;
    const int U = nu + 2, V = nv + 2;
    const int64_t sj = (int64_t)V * n, sa = sj * n, si = sa * U, se = si * n;
    const int tid = threadIdx.x;
    for (int p = tid; p < n * n * n; p += blockDim.x) {
        const int i = p / (n * n), j = (p / n) % n, k = p % n;
        blk[p] = (double)f[e * se + i * si + a * sa + j * sj + b * n + k];
    }
    __syncthreads();
    const double *Lx = lx + (int64_t)le * n * fx;   // [i][p]
    const double *Lu = lu + (int64_t)la * n * fu;   // [j][q]
    const double *Lv = lv + (int64_t)lb * n * fv;   // [k][r]
    for (int p = tid; p < fx * n * n; p += blockDim.x) {
        const int px = p / (n * n), j = (p / n) % n, k = p % n;
        double s = __dmul_rn(Lx[px], blk[j * n + k]);
        for (int i = 1; i < n; ++i) s = __dadd_rn(s, __dmul_rn(Lx[i * fx + px], blk[(i * n + j) * n + k]));
        g1[p] = s;
    }
    __syncthreads();
    for (int p = tid; p < fx * fu * n; p += blockDim.x) {
        const int px = p / (fu * n), q = (p / n) % fu, k = p % n;
        double s = __dmul_rn(Lu[q], g1[(px * n) * n + k]);
        for (int j = 1; j < n; ++j) s = __dadd_rn(s, __dmul_rn(Lu[j * fu + q], g1[(px * n + j) * n + k]));
        g2[p] = s;
    }
    __syncthreads();
    const int64_t o_r = 1, o_b = fv, o_q = (int64_t)ev * fv, o_a = o_q * fu, o_p = o_a * eu,
                  o_e = o_p * fx;
    for (int p = tid; p < fx * fu * fv; p += blockDim.x) {
        const int px = p / (fu * fv), q = (p / fv) % fu, r = p % fv;
        const double *g = g2 + (px * fu + q) * n;
        double s = __dmul_rn(Lv[r], g[0]);
        for (int k = 1; k < n; ++k) s = __dadd_rn(s, __dmul_rn(Lv[k * fv + r], g[k]));
        out[le * o_e + px * o_p + la * o_a + q * o_q + lb * o_b + r * o_r] = s;
    }
}

int check_dims(int precision, int nx, int nu, int nv, int n) {
    if (precision != VL_FP64 && precision != VL_FP32)
        return fail(VL_ERR_INVALID, "precision must be VL_FP64 or VL_FP32");
    if (nx < 1 || nu < 1 || nv < 1 || n < 1) return fail(VL_ERR_INVALID, "empty grid");
    return VL_OK;
}

int grid_for(int64_t total) {
    int64_t g = (total + 255) / 256;
    if (g > 148 * 64) g = 148 * 64;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

extern "C" {

VL_API int vl_initial_state(void *f, int32_t prec, int32_t nx, int32_t nu, int32_t nv, int32_t n,
                            const double *pol, const double *mx, const double *cx,
                            const double *sx, const double *vre, const double *vim, double scale,
                            void *stream) {
    if (!f || !pol) return fail(VL_ERR_INVALID, "null argument");
    if (vre && (!vim || !cx || !sx)) return fail(VL_ERR_INVALID, "mode needs vim, cx and sx");
    if (int rc = check_dims(prec, nx, nu, nv, n)) return rc;
    const int64_t vel = (int64_t)(nu + 2) * n * (nv + 2) * n;
    const int64_t total = (int64_t)(nx + 2) * n * vel;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (prec == VL_FP64)
        initial_state_kernel<double><<<grid_for(total), 256, 0, s>>>(
            static_cast<double *>(f), pol, mx, cx, sx, vre, vim, scale, vel, total);
    else
        initial_state_kernel<float><<<grid_for(total), 256, 0, s>>>(
            static_cast<float *>(f), pol, mx, cx, sx, vre, vim, scale, vel, total);
    return check("initial_state_kernel");
}

VL_API int vl_smooth_edges(void *f, int32_t prec, int32_t nx, int32_t nu, int32_t nv, int32_t n,
                           void *stream) {
    if (!f) return fail(VL_ERR_INVALID, "null argument");
    if (int rc = check_dims(prec, nx, nu, nv, n)) return rc;
    // a pass writes face node 0 (n - 1) and reads the neighbour's node n - 1 (0): with a single
    // node per element both are the same plane and the in-place pass would race
    if (n < 2) return fail(VL_ERR_UNSUPPORTED, "smooth_edges needs at least 2 nodes per element");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t total = (int64_t)nx * nu * nv * n * n;
    for (int axis = 0; axis < 3; ++axis)
        for (int side = 0; side < 2; ++side) {
            if (prec == VL_FP64)
                smooth_pass_kernel<double><<<grid_for(total), 256, 0, s>>>(static_cast<double *>(f),
                                                                           axis, side, nx, nu, nv, n);
            else
                smooth_pass_kernel<float><<<grid_for(total), 256, 0, s>>>(static_cast<float *>(f),
                                                                          axis, side, nx, nu, nv, n);
            const int rc = check("smooth_pass_kernel");
            if (rc) return rc;
        }
    return VL_OK;
}

VL_API int vl_interpolate(const void *f, int32_t prec, int32_t nx, int32_t nu, int32_t nv,
                          int32_t n, const int32_t *lims, const double *ell_x, const double *ell_u,
                          const double *ell_v, int32_t fx, int32_t fu, int32_t fv, double *out,
                          void *stream) {
    if (!f || !lims || !ell_x || !ell_u || !ell_v || !out)
        return fail(VL_ERR_INVALID, "null argument");
    if (int rc = check_dims(prec, nx, nu, nv, n)) return rc;
    const int ext[3] = {nx, nu, nv};
    for (int d = 0; d < 3; ++d)
        if (lims[2 * d] < 1 || lims[2 * d + 1] > ext[d] + 1 || lims[2 * d + 1] <= lims[2 * d])
            return fail(VL_ERR_INVALID, "element range outside the interior");
    if (fx < 1 || fu < 1 || fv < 1 || fx > INTERP_MAX_FINE || fu > INTERP_MAX_FINE || fv > INTERP_MAX_FINE)
        return fail(VL_ERR_INVALID, "fine points per element must be in 1..32");
    if (n > INTERP_MAX_N) return fail(VL_ERR_UNSUPPORTED, "order above 10");
    const size_t smem = sizeof(double) * ((size_t)n * n * n + (size_t)fx * n * n + (size_t)fx * fu * n);
    const dim3 grid(lims[5] - lims[4], lims[3] - lims[2], lims[1] - lims[0]);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (prec == VL_FP64) {
        cudaFuncSetAttribute(interpolate_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        interpolate_kernel<double><<<grid, INTERP_THREADS, smem, s>>>(
            static_cast<const double *>(f), nu, nv, n, lims[0], lims[2], lims[4], grid.z, grid.y,
            grid.x, ell_x, ell_u, ell_v, fx, fu, fv, out);
    } else {
        cudaFuncSetAttribute(interpolate_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        interpolate_kernel<float><<<grid, INTERP_THREADS, smem, s>>>(
            static_cast<const float *>(f), nu, nv, n, lims[0], lims[2], lims[4], grid.z, grid.y,
            grid.x, ell_x, ell_u, ell_v, fx, fu, fv, out);
    }
    return check("interpolate_kernel");
}

}  // extern "C"
