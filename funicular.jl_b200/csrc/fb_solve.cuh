// What the triangular solves of rdiv_upper! (src/kernels.jl:90-124) share,
// k <= 64: the plan a one-CTA prep writes (which path solves, and the
// conditioning behind the choice), the layout of the B fragments it builds,
// and the small complex helpers of both.
//
// Paths, picked on the device from cond_1(R) and the conditioning of R's
// 8 x 8 diagonal blocks:
//   inverse:    Y inv(R) as one product (cond_1(R) <= TR_INV_COND_LIMIT);
//   blocked:    X_b = (Y_b - sum_{c<b} X_c R_cb) inv(R_bb) by 8-column blocks,
//               if every diagonal block has cond_1 up to TR_COND_LIMIT;
//   substitute: plain substitution, a thread per row (the reference's ztrsm
//               arithmetic), otherwise.
// Fragments: the inverse path's n-tile t (four columns) holds k-steps
// 0..2t+1 of the real 4 x 8 form of inv(R), 32 doubles a k-step; the blocked
// path's pair (c, b), c <= b, holds the 16 x 16 real form of -R_cb (c < b) or
// inv(R_bb) (c = b) in TR_FRAG doubles. Each lane's MMA B operand is one
// consecutive 8-byte load either way.
#pragma once

#include "fb_common.cuh"

namespace fb {

constexpr int TR_NB = 8;                 // complex columns per block
constexpr int TR_FRAG = 256;             // doubles per block pair: 4 k-steps x 2 n-tiles x 32 lanes
constexpr double TR_COND_LIMIT = 1.0e4;  // cond_1 of a diagonal block above which substitution is used
constexpr int TR_BUF = TR_NB * TR_NB;    // per-warp transpose buffer: 8 rows x 8 complex, swizzled
constexpr double TR_INV_COND_LIMIT = 16.0;  // cond_1(R) up to which Y R^-1 is one product by inv(R)
constexpr int TR_KMAX = 64;
constexpr int TR_PLAN_BYTES = 256;
constexpr int TR_FRAG_DOUBLES = 36 * TR_FRAG;   // the larger of the two fragment sets at k = 64

enum TrsmPath : int { PATH_INVERSE = 0, PATH_BLOCKED = 1, PATH_SUBSTITUTE = 2 };

struct TrsmPlan {
    int path;
    int pad;
    double cond;          // cond_1(R)
    double cond_blocks;   // largest cond_1 of an 8 x 8 diagonal block
};

// Where (row, col) of the 8 x 8 transpose buffer lives. The writes (C layout:
// a quarter warp covers rows 2j, 2j+1 and four consecutive columns) and the
// reads (A layout: a half warp covers rows 4j..4j+3 and two columns) both
// touch eight different 16-byte chunks of a 128-byte line this way.
__device__ __forceinline__ int tbuf_index(int row, int col) {
    return row * TR_NB + ((col + 4 * (row & 1) + 2 * ((row >> 1) & 1)) & 7);
}

__host__ __device__ __forceinline__ int pair_index(int c, int b) { return b * (b + 1) / 2 + c; }

// Entry (kr, nr) of the real 16 x 16 form of a complex 8 x 8 block M:
// kr = 2 i + p (row i of M, part p of the X entry it multiplies),
// nr = 2 j + o (column j of M, part o of the output).
__device__ __forceinline__ double real_form(z64 m, int p, int o) {
    return o == 0 ? (p == 0 ? m.x : -m.y) : (p == 0 ? m.y : m.x);
}

__device__ __forceinline__ z64 zrecip_d(z64 d) {
    double s = 1.0 / fma(d.x, d.x, d.y * d.y);
    return zmake(d.x * s, -d.y * s);
}

// Doubles of the B fragments a path reads: n-tiles of four columns for the
// inverse, 8 x 8 block pairs for the blocked solve.
__host__ __device__ inline int inverse_frag_doubles(int k) {
    const int nt = (k + 3) / 4;
    return 32 * nt * (nt + 1);
}
__host__ __device__ inline int blocked_frag_doubles(int k) {
    const int nb = (k + TR_NB - 1) / TR_NB;
    return nb * (nb + 1) / 2 * TR_FRAG;
}

}  // namespace fb
