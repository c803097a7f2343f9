// The k x k steps of one cholqr2! pass, as device functions that one CTA of
// any size runs: ||G||_F, the Cholesky of the Gram matrix with the shifted
// retry of cholesky_upper (src/panelblas.jl:148-155), and the solve plan of
// the triangular solve (inv(R), the conditioning, the path and its B
// fragments). The chain's one-CTA kernels and the persistent batch kernel
// both call them, so a factor is computed the same way in either.
#pragma once

#include "fb_solve.cuh"

namespace fb {

// Fixed-order sum over the CTA: warp shuffle tree, then warp 0 over the
// warps. scratch: 33 doubles of shared memory.
__device__ inline double block_sum(double v, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double total = 0.0;
    if (warp == 0) {
        double w = lane < nwarps ? scratch[lane] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) w += __shfl_down_sync(0xffffffffu, w, off);
        if (lane == 0) scratch[32] = w;
    }
    __syncthreads();
    total = scratch[32];
    return total;
}

// ||G||_F over the full Hermitian matrix that the upper triangle g(i, j),
// i <= j, stands for.
template <class LoadG>
__device__ double hermitian_fro(LoadG g, int k, double* scratch) {
    const int tid = threadIdx.x, nt = blockDim.x, kk = k * k;
    double part = 0.0;
    for (int e = tid; e < kk; e += nt) {
        int i = e / k, j = e - i * k;
        if (i <= j) {
            z64 v = g(i, j);
            double a2 = fma(v.x, v.x, v.y * v.y);
            part += (i == j) ? a2 : 2.0 * a2;
        }
    }
    return sqrt(block_sum(part, scratch));
}

// Right-looking Cholesky of the Hermitian matrix g (upper triangle read)
// into W, row-major k x k, upper triangle. Pivot test as LAPACK's zpotrf
// makes it: the factorization fails as soon as a pivot is not > 0 (this also
// catches NaN). On failure the matrix is reloaded with s = 11 N k eps ||G||_F
// added to the diagonal and factored again; a second failure is reported,
// not shifted further. forced_u > 0 instead shifts once, unconditionally, by
// s = 11 (N k + k (k+1)) forced_u ||G||_F (the shifted CholeskyQR3). Returns
// whether a factor was found; shifted and shift say which matrix it is of.
template <class LoadG>
__device__ bool factor_shifted(LoadG g, int k, int64_t N, double gnorm, double forced_u, z64* W, bool& shifted,
                               double& shift) {
    const int tid = threadIdx.x, nt = blockDim.x, kk = k * k;
    shifted = false;
    shift = 0.0;
    bool ok = false;
    if (forced_u > 0.0) {
        shifted = true;
        shift = 11.0 * ((double)N * (double)k + (double)k * (double)(k + 1)) * forced_u * gnorm;
    }
    const int attempts = forced_u > 0.0 ? 1 : 2;
    for (int attempt = 0; attempt < attempts && !ok; ++attempt) {
        if (attempt == 1) {
            shifted = true;
            shift = 11.0 * (double)N * (double)k * 2.220446049250313e-16 * gnorm;
        }
        __syncthreads();
        for (int e = tid; e < kk; e += nt) {
            int i = e / k, j = e - i * k;
            z64 v = zmake(0.0, 0.0);
            if (i <= j) {
                v = g(i, j);
                if (i == j) v = zmake(v.x + shift, 0.0);
            }
            W[e] = v;
        }
        ok = true;
        for (int j = 0; j < k; ++j) {
            __syncthreads();
            const double d = W[j * k + j].x;
            if (!(d > 0.0)) { ok = false; break; }
            const double rj = sqrt(d);
            const double inv = 1.0 / rj;
            for (int l = j + 1 + tid; l < k; l += nt) {
                z64 v = W[j * k + l];
                W[j * k + l] = zmake(v.x * inv, v.y * inv);
            }
            __syncthreads();
            if (tid == 0) W[j * k + j] = zmake(rj, 0.0);
            // The trailing upper triangle: a warp per row m, its lanes along
            // the row's columns l >= m (each entry updated once per step, so
            // the order across entries does not reach the bits).
            const int warp = tid >> 5, lane = tid & 31, nwarps = nt >> 5;
            for (int m = j + 1 + warp; m < k; m += nwarps) {
                const z64 a = W[j * k + m];
                for (int l = m + lane; l < k; l += 32) {
                    const z64 b = W[j * k + l];
                    z64 w = W[m * k + l];
                    // w -= conj(a) * b
                    w.x = fma(-a.x, b.x, w.x);
                    w.x = fma(-a.y, b.y, w.x);
                    w.y = fma(-a.x, b.y, w.y);
                    w.y = fma(a.y, b.x, w.y);
                    W[m * k + l] = w;
                }
            }
        }
        __syncthreads();
    }
    return ok;
}

// Row stride of the prep's KP x KP matrices in shared memory (one complex
// of padding against bank conflicts).
constexpr int TR_PREP_LD = TR_KMAX + 1;

// The solve plan of an upper triangular R, k <= 64: Rs holds R padded with
// the identity to KP x KP (KP = k rounded up to 8), row stride TR_PREP_LD;
// Xs is zeroed, same shape; both are complete (the caller synchronized).
// Computes inv(R) into Xs by rows from the bottom (every column of a row at
// once, four threads to a column sharing the dot product), the 1-norm
// condition numbers of R and of its 8 x 8 diagonal blocks, the path, and the
// chosen path's B fragments into frag.
__device__ inline void solve_plan(const z64* Rs, z64* Xs, int k, TrsmPlan* plan, double* __restrict__ frag) {
    constexpr int LD = TR_PREP_LD;
    __shared__ z64 dinv[TR_KMAX];
    __shared__ double colr[TR_KMAX], coli[TR_KMAX];
    __shared__ double bcolr[TR_KMAX], bcoli[TR_KMAX];
    __shared__ int path;
    const int tid = threadIdx.x;
    const int KP = (k + TR_NB - 1) / TR_NB * TR_NB;
    for (int j = tid; j < KP; j += blockDim.x) dinv[j] = zrecip_d(Rs[j * LD + j]);
    __syncthreads();
    // Row i of inv(R): X[i][j] = (delta_ij - sum_{i<l<=j} R[i][l] X[l][j]) / R[i][i].
    for (int i = KP - 1; i >= 0; --i) {
        for (int base = 0; base < 4 * KP; base += blockDim.x) {
            const int t = base + tid, col = t >> 2, part = t & 3;
            z64 acc = zmake(0.0, 0.0);
            if (col < KP && col >= i)
                for (int l = i + 1 + part; l <= col; l += 4) zmac(acc, Rs[i * LD + l], Xs[l * LD + col]);
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 2);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 2);
            if (col < KP && col >= i && part == 0) {
                const z64 rhs = zmake((i == col ? 1.0 : 0.0) - acc.x, -acc.y);
                Xs[i * LD + col] = zmul(rhs, dinv[i]);
            }
        }
        __syncthreads();
    }
    // 1-norms of R's own columns and of inv(R)'s, and of the columns of
    // their 8 x 8 diagonal blocks: a thread per column, each sum in row order.
    for (int c = tid; c < KP; c += blockDim.x) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i <= c; ++i) {
            a += hypot(Rs[i * LD + c].x, Rs[i * LD + c].y);
            b += hypot(Xs[i * LD + c].x, Xs[i * LD + c].y);
        }
        colr[c] = c < k ? a : 0.0;
        coli[c] = c < k ? b : 0.0;
        double cr = 0.0, ci = 0.0;
        for (int i = TR_NB * (c / TR_NB); i <= c; ++i) {
            cr += hypot(Rs[i * LD + c].x, Rs[i * LD + c].y);
            ci += hypot(Xs[i * LD + c].x, Xs[i * LD + c].y);
        }
        bcolr[c] = cr;
        bcoli[c] = ci;
    }
    __syncthreads();
    if (tid == 0) {
        double nr = 0.0, ni = 0.0;
        for (int j = 0; j < KP; ++j) {
            nr = fmax(nr, colr[j]);
            ni = fmax(ni, coli[j]);
        }
        const double cond = nr * ni;
        double worst = 0.0;
        for (int b = 0; b < KP / TR_NB; ++b) {
            double br = 0.0, bi = 0.0;
            for (int j = TR_NB * b; j < TR_NB * b + TR_NB; ++j) {
                br = fmax(br, bcolr[j]);
                bi = fmax(bi, bcoli[j]);
            }
            worst = fmax(worst, br * bi);
        }
        int p = PATH_SUBSTITUTE;
        if (cond <= TR_INV_COND_LIMIT) p = PATH_INVERSE;
        else if (worst <= TR_COND_LIMIT) p = PATH_BLOCKED;
        path = p;
        plan->path = p;
        plan->cond = cond;
        plan->cond_blocks = worst;
    }
    __syncthreads();
    if (path == PATH_INVERSE) {
        const int NT = (k + 3) / 4;
        for (int e = tid; e < 32 * NT * (NT + 1); e += blockDim.x) {
            int t = 0;
            while (32 * (t + 1) * (t + 2) <= e) ++t;
            const int f = e - 32 * t * (t + 1);
            const int s = f >> 5, lane = f & 31;
            const int i = 2 * s + ((lane & 3) >> 1), p = lane & 1;
            const int j = 4 * t + ((lane >> 2) >> 1), o = (lane >> 2) & 1;
            frag[e] = (i <= j) ? real_form(Xs[i * LD + j], p, o) : 0.0;
        }
    } else if (path == PATH_BLOCKED) {
        const int NBLK = KP / TR_NB;
        const int npairs = NBLK * (NBLK + 1) / 2;
        for (int e = tid; e < npairs * TR_FRAG; e += blockDim.x) {
            const int pr = e / TR_FRAG, f = e - pr * TR_FRAG;
            int b = 0;
            while (pair_index(0, b + 1) <= pr) ++b;
            const int c = pr - pair_index(0, b);
            const int lane = f & 31, st_ = f >> 5, s = st_ >> 1, t = st_ & 1;
            const int kr = 4 * s + (lane & 3), nr = 8 * t + (lane >> 2);
            const int i = TR_NB * c + (kr >> 1), p = kr & 1, j = TR_NB * b + (nr >> 1), o = nr & 1;
            // -R_cb off the diagonal; inv(R_bb), which is inv(R)'s own diagonal block, on it.
            frag[e] = (c < b) ? -real_form(Rs[i * LD + j], p, o) : real_form(Xs[i * LD + j], p, o);
        }
    }
}

}  // namespace fb
