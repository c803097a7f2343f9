// The matrix-free operator of the streamed range finder (a complex-shifted
// 3-D Laplacian on a 342^3 grid): G = -Lap_7 + shift I on an nx x ny x nz grid, applied to the columns of a
// device panel, the panel-capable mul! that apply_operator! hands a whole
// resident panel to (src/operator.jl:80-87). Grid point (x, y, z) is row
// x + nx (y + ny z); the 7-point Laplacian has unit spacing and zero
// (Dirichlet) values outside the grid:
//   (G v)_p = (6 + shift) v_p - sum of the six neighbours of p.
// HBM-bound: 32 bytes per entry (read once, write once) when the neighbours
// are read from DRAM once. Two kernels: by 2.5-D tiles (the default), and a
// thread per output entry for column counts past the grid limit.
#include "fb_common.cuh"

namespace fb {

// Blocks walk grid lines (fixed y, z) and threads the points of a line, so
// the index arithmetic is one 32-bit division per line.
__global__ void __launch_bounds__(128) laplace7_kernel(z64* __restrict__ Y, int64_t ldy, const z64* __restrict__ X,
                                                       int64_t ldx, int nx, int ny, int nz, int cols, z64 shift) {
    const int64_t plane = (int64_t)nx * ny;
    const int lines = ny * nz;
    const double dr = 6.0 + shift.x, di = shift.y;
    for (int c = blockIdx.y; c < cols; c += gridDim.y) {
        const z64* x = X + (int64_t)c * ldx;
        z64* y = Y + (int64_t)c * ldy;
        for (int line = blockIdx.x; line < lines; line += gridDim.x) {
            const int zi = line / ny, yi = line - zi * ny;
            const int64_t base = (int64_t)line * nx;
            for (int xi = threadIdx.x; xi < nx; xi += blockDim.x) {
                const int64_t p = base + xi;
                const z64 v = x[p];
                z64 s = zmake(0.0, 0.0);
                if (xi > 0) { const z64 u = x[p - 1]; s.x += u.x; s.y += u.y; }
                if (xi < nx - 1) { const z64 u = x[p + 1]; s.x += u.x; s.y += u.y; }
                if (yi > 0) { const z64 u = x[p - nx]; s.x += u.x; s.y += u.y; }
                if (yi < ny - 1) { const z64 u = x[p + nx]; s.x += u.x; s.y += u.y; }
                if (zi > 0) { const z64 u = x[p - plane]; s.x += u.x; s.y += u.y; }
                if (zi < nz - 1) { const z64 u = x[p + plane]; s.x += u.x; s.y += u.y; }
                y[p] = zmake(dr * v.x - di * v.y - s.x, dr * v.y + di * v.x - s.y);
            }
        }
    }
}

// The same operator by 2.5-D tiles: a block owns a 32 x 8 tile of an x-y
// plane of one column and marches it along a range of z. Each thread keeps
// its point's values at z - 1, z and z + 1 in registers, with the plane at
// z + 2 already loading (one new plane read a step, two steps ahead of its
// use), and the x and y neighbours come from the current plane staged in
// shared memory with a one-point halo (its edge points read from L2, where
// the neighbouring tiles marching beside this one have brought them). Every
// input is read from DRAM about once. The z range of a column is cut into
// zchunks pieces, enough for the grid to fill the GPU when there are few
// columns.
constexpr int LT_X = 32, LT_Y = 8;

__global__ void __launch_bounds__(LT_X * LT_Y)
laplace7_tiled_kernel(z64* __restrict__ Y, int64_t ldy, const z64* __restrict__ X, int64_t ldx, int nx, int ny,
                      int nz, z64 shift, int zchunks) {
    __shared__ z64 tile[LT_Y + 2][LT_X + 2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int gx = blockIdx.x * LT_X + tx, gy = blockIdx.y * LT_Y + ty;
    const int c = blockIdx.z / zchunks, zc = blockIdx.z - c * zchunks;
    const int z0 = (int)((int64_t)nz * zc / zchunks), z1 = (int)((int64_t)nz * (zc + 1) / zchunks);
    const z64* x = X + (int64_t)c * ldx;
    z64* y = Y + (int64_t)c * ldy;
    const int64_t plane = (int64_t)nx * ny;
    const bool inside = gx < nx && gy < ny;
    const int64_t col_off = (int64_t)gy * nx + gx;
    const double dr = 6.0 + shift.x, di = shift.y;
    const z64 zero = zmake(0.0, 0.0);
    auto at = [&](int xx, int yy, int zz) -> z64 {
        return (xx >= 0 && xx < nx && yy >= 0 && yy < ny && zz >= 0 && zz < nz)
                   ? x[(int64_t)zz * plane + (int64_t)yy * nx + xx] : zero;
    };
    auto plane_at = [&](int zz) -> z64 { return (inside && zz >= 0 && zz < nz) ? x[(int64_t)zz * plane + col_off] : zero; };
    z64 below = plane_at(z0 - 1);
    z64 cur = plane_at(z0);
    z64 above = plane_at(z0 + 1);
    z64 ahead = plane_at(z0 + 2);
    // Halo: the columns x0 - 1 and x0 + 32 (lanes 0..7 of the first two
    // warps) and the rows y0 - 1 and y0 + 8 (the next two warps); each such
    // thread loads its halo point one plane ahead.
    int hx = -2, hy = -2, hr = 0, hc = 0;
    if (ty == 0 && tx < LT_Y) { hx = blockIdx.x * LT_X - 1; hy = blockIdx.y * LT_Y + tx; hr = tx + 1; hc = 0; }
    if (ty == 1 && tx < LT_Y) { hx = blockIdx.x * LT_X + LT_X; hy = blockIdx.y * LT_Y + tx; hr = tx + 1; hc = LT_X + 1; }
    if (ty == 2) { hx = gx; hy = blockIdx.y * LT_Y - 1; hr = 0; hc = tx + 1; }
    if (ty == 3) { hx = gx; hy = blockIdx.y * LT_Y + LT_Y; hr = LT_Y + 1; hc = tx + 1; }
    const bool halo = hx != -2;
    z64 hval = halo ? at(hx, hy, z0) : zero;
    for (int z = z0; z < z1; ++z) {
        tile[ty + 1][tx + 1] = cur;
        if (halo) tile[hr][hc] = hval;
        __syncthreads();
        if (inside) {
            const z64 a = tile[ty + 1][tx], b = tile[ty + 1][tx + 2], d = tile[ty][tx + 1], e = tile[ty + 2][tx + 1];
            const double sx = a.x + b.x + d.x + e.x + below.x + above.x;
            const double sy = a.y + b.y + d.y + e.y + below.y + above.y;
            y[(int64_t)z * plane + col_off] = zmake(dr * cur.x - di * cur.y - sx, dr * cur.y + di * cur.x - sy);
        }
        __syncthreads();
        below = cur;
        cur = above;
        above = ahead;
        ahead = plane_at(z + 3);
        if (halo) hval = at(hx, hy, z + 1);
    }
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_zlaplace7_apply(fb_z128* Y, int64_t ldy, const fb_z128* X, int64_t ldx, int nx, int ny, int nz, int cols,
                       fb_z128 shift, fb_queue_t queue) {
    if (nx < 1 || ny < 1 || nz < 1 || cols < 0) {
        set_error(FB_EINVAL, "fb_zlaplace7_apply: the grid needs positive sizes and cols >= 0, got %d x %d x %d, "
                  "%d columns", nx, ny, nz, cols);
        return FB_EINVAL;
    }
    const int64_t n = (int64_t)nx * ny * nz;
    if (cols == 0) return FB_OK;
    if (!Y || !X) { set_error(FB_EINVAL, "fb_zlaplace7_apply: NULL matrix"); return FB_EINVAL; }
    if (ldy < n || ldx < n) {
        set_error(FB_EDIM, "fb_zlaplace7_apply: leading dimensions %lld, %lld below the %lld grid points",
                  (long long)ldy, (long long)ldx, (long long)n);
        return FB_EDIM;
    }
    if (((uintptr_t)Y | (uintptr_t)X) & 15) { set_error(FB_EINVAL, "fb_zlaplace7_apply: pointers must be 16-byte aligned"); return FB_EINVAL; }
    // Y and X must not overlap: every output reads seven inputs.
    const char* y0 = reinterpret_cast<const char*>(Y);
    const char* x0 = reinterpret_cast<const char*>(X);
    const size_t ybytes = ((size_t)(cols - 1) * ldy + n) * 16, xbytes = ((size_t)(cols - 1) * ldx + n) * 16;
    if (y0 < x0 + xbytes && x0 < y0 + ybytes) {
        set_error(FB_EINVAL, "fb_zlaplace7_apply: the output overlaps the input");
        return FB_EINVAL;
    }
    if ((int64_t)ny * nz > INT32_MAX) { set_error(FB_ENOTSUP, "fb_zlaplace7_apply: ny * nz must fit in 32 bits"); return FB_ENOTSUP; }
    const int64_t tiles = (int64_t)((nx + LT_X - 1) / LT_X) * ((ny + LT_Y - 1) / LT_Y);
    // z pieces: enough blocks for eight a SM, each piece at least 16 planes.
    int64_t zchunks = ((int64_t)sm_count() * 8 + tiles * cols - 1) / (tiles * cols);
    if (zchunks > nz / 16) zchunks = nz / 16;
    if (zchunks < 1) zchunks = 1;
    if (cols * zchunks <= 65535 && (ny + LT_Y - 1) / LT_Y <= 65535) {
        const dim3 grid((unsigned)((nx + LT_X - 1) / LT_X), (unsigned)((ny + LT_Y - 1) / LT_Y),
                        (unsigned)(cols * zchunks));
        laplace7_tiled_kernel<<<grid, dim3(LT_X, LT_Y), 0, stream_of(queue)>>>(
            reinterpret_cast<z64*>(Y), ldy, reinterpret_cast<const z64*>(X), ldx, nx, ny, nz, zmake(shift.re, shift.im),
            (int)zchunks);
        FB_LAUNCHED("laplace7_tiled_kernel");
        return FB_OK;
    }
    // Sixteen blocks per SM, every block walking the columns in the same order
    // and the lines of a column in a grid-strided sweep: the lines in flight
    // at one time span a few planes of one column, so the z neighbours of a
    // line are still in L2 when it is computed.
    const int64_t gy = 1;
    int64_t gx = (int64_t)sm_count() * 16;
    if (gx > (int64_t)ny * nz) gx = (int64_t)ny * nz;
    if (gx < 1) gx = 1;
    laplace7_kernel<<<dim3((unsigned)gx, (unsigned)gy), 128, 0, stream_of(queue)>>>(
        reinterpret_cast<z64*>(Y), ldy, reinterpret_cast<const z64*>(X), ldx, nx, ny, nz, cols,
        zmake(shift.re, shift.im));
    FB_LAUNCHED("laplace7_kernel");
    return FB_OK;
}

}  // extern "C"
