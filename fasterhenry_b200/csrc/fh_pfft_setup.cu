// Device part of the precorrected-FFT set-up (pfft/mod.rs:332-460,
// grid.rs:100-216, near.rs:114-401 of the reference):
//
//   * projection: thread per filament.  A composite Gauss-Legendre rule over
//     the filament's length, width and height (pieces no longer than h, the
//     order from the 1e-10 / 12 table at the near-field distance) is
//     interpolated onto the (order+1)^3 Lagrange stencil of every node and
//     summed, node by node in the rule's order, into a dense box of grid
//     points private to the filament; the touched points, in ascending grid
//     index, are the filament's row of W.  Its transpose (by grid point, then
//     filament) comes from a stable radix sort.
//   * grid approximation of every near pair, sum_g sum_h W_ig W_jh K(g - h):
//     block per row i, the row's projection staged in shared memory, warp
//     per partner j, lanes over j's projection, a fixed reduction tree.
//     K(d) = 1 / (h |d|) (zero at the origin) is tabulated once over the
//     offsets the pairs reach.
//   * the near-field matrix: exact - mu0/4pi cos approximation per pair,
//     mirrored into full rows ascending in column by one radix sort.
//
// Every result is deterministic: each filament's sums run in a fixed order
// on one thread, each pair's on one warp with a fixed shuffle tree.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "fh_device.cuh"
#include "fh_pfft.h"

namespace fhb {
namespace {

constexpr double kMu0Over4PiS = 1.0e-7;

struct ProjConst {
    double x[kProjectionMaxOrder + 1][kProjectionMaxOrder];
    double w[kProjectionMaxOrder + 1][kProjectionMaxOrder];
    double threshold[kProjectionMaxOrder];
};
__constant__ ProjConst c_proj;
bool g_proj_uploaded[64] = {false};
std::mutex g_proj_mu;

struct GridArgs {
    double origin[3];
    double spacing;
    int64_t dims[3];
    int m;
};

// First stencil plane along axis a for coordinate x (grid.rs:100-120).
__host__ __device__ inline int64_t stencil_first(const GridArgs &g, int a, double x) {
    const double u = (x - g.origin[a]) / g.spacing;
    const double f = floor(u - 0.5 * g.m) + 1.0;
    int64_t first = f > 0.0 ? (int64_t)f : 0;
    const int64_t last = g.dims[a] - g.m;
    return first < last ? first : last;
}

// The m Lagrange weights of the stencil starting at `first`.
__device__ inline void stencil_weights(const GridArgs &g, int a, double x, int64_t first, double *w) {
    const double t = (x - g.origin[a]) / g.spacing - (double)first;
    for (int k = 0; k < g.m; ++k) {
        double v = 1.0;
        for (int l = 0; l < g.m; ++l)
            if (l != k) v *= (t - (double)l) / ((double)k - (double)l);
        w[k] = v;
    }
}

// OrderTable(1e-10, 12).order_for (gauss.rs:123-136); 0 when none suffices.
__device__ inline int projection_order(double half, double distance) {
    if (half <= 0.0) return 1;
    if (isnan(distance) || distance <= 0.0) return 0;
    const double delta = distance / half;
    for (int k = 0; k < kProjectionMaxOrder; ++k)
        if (delta >= c_proj.threshold[k]) return k + 1;
    return 0;
}

// Per filament: its box of grid points (lo corner, dims) and scratch offset.
struct Box {
    int64_t lo[3];
    int32_t dims[3];
    int32_t pad;
    int64_t offset;
};

__global__ void __launch_bounds__(128) project_kernel(const fh_filament *__restrict__ fil, int64_t n, GridArgs g,
                                                      double far, const Box *__restrict__ boxes,
                                                      double *__restrict__ scratch, uint8_t *__restrict__ touched,
                                                      int64_t *__restrict__ counts, int *__restrict__ overflow) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const fh_filament f = fil[i];
    const Box b = boxes[i];
    const double *axes[3] = {f.dir_length, f.dir_width, f.dir_height};
    const double extents[3] = {f.length, f.width, f.height};
    double corner[3];
    for (int k = 0; k < 3; ++k) corner[k] = f.start[k] - 0.5 * f.width * f.dir_width[k] - 0.5 * f.height * f.dir_height[k];
    int64_t pieces[3];
    int order[3];
    double piece[3];
    for (int d = 0; d < 3; ++d) {
        const double p = ceil(extents[d] / g.spacing);
        pieces[d] = p > 1.0 ? (int64_t)p : 1;
        piece[d] = extents[d] / (double)pieces[d];
        const int o = projection_order(0.5 * piece[d], far);
        order[d] = o == 0 ? kProjectionMaxOrder : o;
    }
    const double inverse_area = 1.0 / (f.width * f.height);
    const int m = g.m;
    double *box = scratch + b.offset;
    uint8_t *hit = touched + b.offset;
    double wx[16], wy[16], wz[16];
    for (int64_t p0 = 0; p0 < pieces[0]; ++p0)
        for (int q0 = 0; q0 < order[0]; ++q0) {
            const double a0 = (double)p0 * piece[0], b0 = (double)(p0 + 1) * piece[0];
            const double h0 = 0.5 * (b0 - a0);
            const double s = 0.5 * (a0 + b0) + h0 * c_proj.x[order[0]][q0], ws = h0 * c_proj.w[order[0]][q0];
            for (int64_t p1 = 0; p1 < pieces[1]; ++p1)
                for (int q1 = 0; q1 < order[1]; ++q1) {
                    const double a1 = (double)p1 * piece[1], b1 = (double)(p1 + 1) * piece[1];
                    const double h1 = 0.5 * (b1 - a1);
                    const double t = 0.5 * (a1 + b1) + h1 * c_proj.x[order[1]][q1], wt = h1 * c_proj.w[order[1]][q1];
                    for (int64_t p2 = 0; p2 < pieces[2]; ++p2)
                        for (int q2 = 0; q2 < order[2]; ++q2) {
                            const double a2 = (double)p2 * piece[2], b2 = (double)(p2 + 1) * piece[2];
                            const double h2 = 0.5 * (b2 - a2);
                            const double u = 0.5 * (a2 + b2) + h2 * c_proj.x[order[2]][q2];
                            const double wu = h2 * c_proj.w[order[2]][q2];
                            double r[3];
                            for (int k = 0; k < 3; ++k)
                                r[k] = corner[k] + s * axes[0][k] + t * axes[1][k] + u * axes[2][k];
                            const double weight = ws * wt * wu * inverse_area;
                            const int64_t fx = stencil_first(g, 0, r[0]), fy = stencil_first(g, 1, r[1]),
                                          fz = stencil_first(g, 2, r[2]);
                            const int64_t ox = fx - b.lo[0], oy = fy - b.lo[1], oz = fz - b.lo[2];
                            if (ox < 0 || oy < 0 || oz < 0 || ox + m > b.dims[0] || oy + m > b.dims[1] ||
                                oz + m > b.dims[2]) {
                                atomicExch(overflow, 1);  // never writes outside the box
                                continue;
                            }
                            stencil_weights(g, 0, r[0], fx, wx);
                            stencil_weights(g, 1, r[1], fy, wy);
                            stencil_weights(g, 2, r[2], fz, wz);
                            for (int ii = 0; ii < m; ++ii)
                                for (int jj = 0; jj < m; ++jj) {
                                    const int64_t row = ((ox + ii) * b.dims[1] + (oy + jj)) * b.dims[2] + oz;
                                    const double lxy = weight * wx[ii] * wy[jj];
                                    for (int kk = 0; kk < m; ++kk) {
                                        box[row + kk] += lxy * wz[kk];
                                        hit[row + kk] = 1;
                                    }
                                }
                        }
                }
        }
    const int64_t cells = (int64_t)b.dims[0] * b.dims[1] * b.dims[2];
    int64_t c = 0;
    for (int64_t k = 0; k < cells; ++k) c += hit[k];
    counts[i] = c;
}

// Writes the touched points of each box, ascending grid index, with their
// filament, and the filament's grid-coordinate bounds.
__global__ void __launch_bounds__(128) project_emit_kernel(int64_t n, GridArgs g, const Box *__restrict__ boxes,
                                                           const double *__restrict__ scratch,
                                                           const uint8_t *__restrict__ touched,
                                                           const int64_t *__restrict__ off, uint32_t *__restrict__ idx,
                                                           double *__restrict__ w, int32_t *__restrict__ owner,
                                                           int32_t *__restrict__ lohi) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Box b = boxes[i];
    int64_t o = off[i];
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {0, 0, 0};
    for (int32_t x = 0; x < b.dims[0]; ++x)
        for (int32_t y = 0; y < b.dims[1]; ++y)
            for (int32_t z = 0; z < b.dims[2]; ++z) {
                const int64_t cell = ((int64_t)x * b.dims[1] + y) * b.dims[2] + z;
                if (!touched[b.offset + cell]) continue;
                const int64_t gx = b.lo[0] + x, gy = b.lo[1] + y, gz = b.lo[2] + z;
                idx[o] = (uint32_t)((gx * g.dims[1] + gy) * g.dims[2] + gz);
                w[o] = scratch[b.offset + cell];
                owner[o] = (int32_t)i;
                ++o;
                const int32_t p[3] = {(int32_t)gx, (int32_t)gy, (int32_t)gz};
                for (int a = 0; a < 3; ++a) {
                    lo[a] = min(lo[a], p[a]);
                    hi[a] = max(hi[a], p[a]);
                }
            }
    for (int a = 0; a < 3; ++a) {
        lohi[6 * i + a] = lo[a];
        lohi[6 * i + 3 + a] = hi[a];
    }
}

__global__ void gather_spread_kernel(const uint32_t *__restrict__ pos, const int32_t *__restrict__ owner,
                                     const double *__restrict__ w, int64_t count, uint32_t *__restrict__ fil_out,
                                     double *__restrict__ w_out) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
        fil_out[k] = (uint32_t)owner[pos[k]];
        w_out[k] = w[pos[k]];
    }
}

__global__ void count_keys_kernel(const uint32_t *__restrict__ keys, int64_t count, unsigned long long *__restrict__ c) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&c[keys[k]], 1ull);
}

__global__ void iota_kernel(uint32_t *__restrict__ v, int64_t count) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x)
        v[k] = (uint32_t)k;
}

// Largest offsets between a filament's projection and its partners'
// (near.rs:244-253): per pair, max(hi_j - lo_i, hi_i - lo_j, 0) per axis.
__global__ void reach_kernel(const int2 *__restrict__ pairs, int64_t np, const int32_t *__restrict__ lohi,
                             int *__restrict__ reach) {
    int r[3] = {0, 0, 0};
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < np; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = pairs[k].x, j = pairs[k].y;
        for (int a = 0; a < 3; ++a)
            r[a] = max(r[a], max(lohi[6 * j + 3 + a] - lohi[6 * i + a], lohi[6 * i + 3 + a] - lohi[6 * j + a]));
    }
    for (int a = 0; a < 3; ++a) atomicMax(&reach[a], r[a]);
}

// K(d) = 1 / (h |d|), zero at d = 0, over |d_a| <= reach_a, z fastest (near.rs:114-170).
__global__ void kernel_table_kernel(double *__restrict__ t, int rx, int ry, int rz, double spacing) {
    const int64_t dy = 2 * ry + 1, dz = 2 * rz + 1, total = (int64_t)(2 * rx + 1) * dy * dz;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = k / (dy * dz) - rx, y = (k / dz) % dy - ry, z = k % dz - rz;
        const double r2 = (double)(x * x + y * y + z * z);
        t[k] = r2 == 0.0 ? 0.0 : 1.0 / (spacing * sqrt(r2));
    }
}

constexpr int kPreThreads = 128;
constexpr int kPreChunk = 512;

// Block per row i: grid[k] = sum over j's entries e of w_e sum over i's
// entries s of w_s K(e - s), for the row's pairs k.
__global__ void __launch_bounds__(kPreThreads) precorrect_kernel(
    int64_t n, GridArgs g, const int64_t *__restrict__ pair_off, const int2 *__restrict__ pairs,
    const int64_t *__restrict__ proj_off, const uint32_t *__restrict__ proj_idx, const double *__restrict__ proj_w,
    const double *__restrict__ table, int rx, int ry, int rz, double *__restrict__ grid) {
    __shared__ int32_t sx[kPreChunk], sy[kPreChunk], sz[kPreChunk];
    __shared__ double sw[kPreChunk];
    const int64_t dyz = (int64_t)(2 * ry + 1) * (2 * rz + 1), dz = 2 * rz + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = kPreThreads / 32;
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int64_t k0 = pair_off[i], k1 = pair_off[i + 1];
        if (k0 == k1) continue;
        const int64_t s0 = proj_off[i], s1 = proj_off[i + 1];
        for (int64_t c0 = s0; c0 < s1; c0 += kPreChunk) {
            const int cn = (int)(s1 - c0 < kPreChunk ? s1 - c0 : kPreChunk);
            __syncthreads();
            for (int t = threadIdx.x; t < cn; t += kPreThreads) {
                const int64_t gi = proj_idx[c0 + t];
                sz[t] = (int32_t)(gi % g.dims[2]);
                const int64_t rest = gi / g.dims[2];
                sy[t] = (int32_t)(rest % g.dims[1]);
                sx[t] = (int32_t)(rest / g.dims[1]);
                sw[t] = proj_w[c0 + t];
            }
            __syncthreads();
            for (int64_t k = k0 + warp; k < k1; k += warps) {
                const int j = pairs[k].y;
                double acc = 0.0;
                for (int64_t e = proj_off[j] + lane; e < proj_off[j + 1]; e += 32) {
                    const int64_t ge = proj_idx[e];
                    const int32_t ez = (int32_t)(ge % g.dims[2]);
                    const int64_t rest = ge / g.dims[2];
                    const int32_t ey = (int32_t)(rest % g.dims[1]), ex = (int32_t)(rest / g.dims[1]);
                    const double *base = table + (int64_t)(ex + rx) * dyz + (int64_t)(ey + ry) * dz + (ez + rz);
                    double potential = 0.0;
                    for (int t = 0; t < cn; ++t)
                        potential += sw[t] * base[-((int64_t)sx[t] * dyz + (int64_t)sy[t] * dz + sz[t])];
                    acc += proj_w[e] * potential;
                }
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if (lane == 0) grid[k] = (c0 == s0 ? 0.0 : grid[k]) + acc;
            }
        }
    }
}

// Near-field entries: c = exact - mu0/4pi cos grid, keyed row * n + column;
// the mirrored entry of an off-diagonal pair goes to slot np + k, a diagonal
// pair's mirror slot gets the largest key (sorted past the end).
__global__ void near_entries_kernel(const int2 *__restrict__ pairs, int64_t np, int64_t n,
                                    const double *__restrict__ exact, const double *__restrict__ cosv,
                                    const double *__restrict__ grid, unsigned long long *__restrict__ keys,
                                    double *__restrict__ vals, unsigned long long *__restrict__ row_counts) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < np; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = pairs[k].x, j = pairs[k].y;
        const double c = exact[k] - kMu0Over4PiS * cosv[k] * grid[k];
        keys[k] = (unsigned long long)(i * n + j);
        vals[k] = c;
        atomicAdd(&row_counts[i], 1ull);
        if (i != j) {
            keys[np + k] = (unsigned long long)(j * n + i);
            vals[np + k] = c;
            atomicAdd(&row_counts[j], 1ull);
        } else {
            keys[np + k] = ~0ull;
            vals[np + k] = 0.0;
        }
    }
}

__global__ void near_split_kernel(const unsigned long long *__restrict__ keys, const double *__restrict__ vals,
                                  int64_t count, int64_t n, uint32_t *__restrict__ col, double *__restrict__ val) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
        col[k] = (uint32_t)(keys[k] % (unsigned long long)n);
        val[k] = vals[k];
    }
}

inline unsigned blocks(int64_t work, int threads) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + threads - 1) / threads, 148 * 32));
}

// Scratch freed on scope exit, in stream order.
struct Scratch {
    cudaStream_t s;
    std::vector<void *> p;
    ~Scratch() {
        for (void *q : p) cache_free(q, s);
    }
    template <class T>
    cudaError_t get(T **out, size_t count) {
        void *q = nullptr;
        cudaError_t e = cache_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), s);
        if (e == cudaSuccess) {
            p.push_back(q);
            *out = static_cast<T *>(q);
        }
        return e;
    }
};

template <class T>
cudaError_t persist(T **out, size_t count) {
    return cudaMalloc((void **)out, std::max<size_t>(count, 1) * sizeof(T));
}

fh_status upload_constants(fh_error_info *err) {
    int dev = 0;
    FHB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_proj_mu);
    if (dev < 64 && g_proj_uploaded[dev]) return FH_OK;
    ProjConst c{};
    for (int k = 1; k <= kProjectionMaxOrder; ++k) gauss_rule(k, c.x[k], c.w[k]);
    // OrderTable thresholds: the Bernstein-ellipse ratio for the tolerance at order k.
    const double lg = std::log(1.0 / kProjectionTolerance);
    for (int k = 1; k <= kProjectionMaxOrder; ++k) c.threshold[k - 1] = std::sinh(lg / (2.0 * k));
    FHB_CUDA(cudaMemcpyToSymbol(c_proj, &c, sizeof c));
    if (dev < 64) g_proj_uploaded[dev] = true;
    return FH_OK;
}

}  // namespace

fh_status pfft_device_setup(const PfftSetup &st, const fh_filament *fil, const NearPairs &near, cudaStream_t s,
                            PfftDeviceSetup &out, fh_error_info *err) {
    out = PfftDeviceSetup();
    const int64_t n = st.n;
    if (n == 0) return FH_OK;
    fh_status e = upload_constants(err);
    if (e) return e;
    GridArgs g;
    for (int a = 0; a < 3; ++a) {
        g.origin[a] = st.grid.origin[a];
        g.dims[a] = st.grid.dims[a];
    }
    g.spacing = st.grid.spacing;
    g.m = st.grid.stencil;
    const int64_t G = st.grid.len();
    // Boxes: the stencil planes reachable from the filament's volume.
    std::vector<Box> boxes((size_t)n);
    int64_t scratch_cells = 0;
    for (int64_t i = 0; i < n; ++i) {
        const fh_filament &f = fil[i];
        Box &b = boxes[(size_t)i];
        for (int a = 0; a < 3; ++a) {
            double lo = INFINITY, hi = -INFINITY;
            for (int c = 0; c < 8; ++c) {
                const double x = f.start[a] + ((c & 1) ? f.length * f.dir_length[a] : 0.0) +
                                 ((c & 2) ? 0.5 : -0.5) * f.width * f.dir_width[a] +
                                 ((c & 4) ? 0.5 : -0.5) * f.height * f.dir_height[a];
                lo = std::min(lo, x);
                hi = std::max(hi, x);
            }
            const int64_t first = stencil_first(g, a, lo), last = stencil_first(g, a, hi);
            b.lo[a] = first;
            b.dims[a] = (int32_t)(last - first + g.m);
        }
        b.pad = 0;
        b.offset = scratch_cells;
        scratch_cells += (int64_t)b.dims[0] * b.dims[1] * b.dims[2];
    }
    Scratch tmp{s, {}};
    fh_filament *d_fil;
    Box *d_boxes;
    double *d_scratch;
    uint8_t *d_touched;
    int64_t *d_counts;
    int *d_flag;
    FHB_CUDA(tmp.get(&d_fil, (size_t)n));
    FHB_CUDA(tmp.get(&d_boxes, (size_t)n));
    FHB_CUDA(tmp.get(&d_scratch, (size_t)scratch_cells));
    FHB_CUDA(tmp.get(&d_touched, (size_t)scratch_cells));
    FHB_CUDA(tmp.get(&d_counts, (size_t)n + 1));
    FHB_CUDA(tmp.get(&d_flag, 4));
    FHB_CUDA(cudaMemcpyAsync(d_fil, fil, sizeof(fh_filament) * n, cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemcpyAsync(d_boxes, boxes.data(), sizeof(Box) * n, cudaMemcpyHostToDevice, s));
    FHB_CUDA(cudaMemsetAsync(d_scratch, 0, sizeof(double) * scratch_cells, s));
    FHB_CUDA(cudaMemsetAsync(d_touched, 0, scratch_cells, s));
    FHB_CUDA(cudaMemsetAsync(d_flag, 0, 16, s));
    FHB_CUDA(cudaMemsetAsync(d_counts + n, 0, 8, s));
    project_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(d_fil, n, g, st.radius, d_boxes, d_scratch, d_touched,
                                                               d_counts, d_flag);
    FHB_CUDA(cudaGetLastError());
    // Row offsets of the projection: exclusive sum of the counts.
    FHB_CUDA(persist(&out.proj_off, (size_t)n + 1));
    size_t tb = 0;
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_counts, out.proj_off, (int)(n + 1), s));
    void *d_tb;
    FHB_CUDA(tmp.get((uint8_t **)&d_tb, tb));
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(d_tb, tb, d_counts, out.proj_off, (int)(n + 1), s));
    int flag = 0;
    FHB_CUDA(cudaMemcpyAsync(&out.entries, out.proj_off + n, 8, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaMemcpyAsync(&flag, d_flag, 4, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    if (flag) return fail(err, FH_ERR_PFFT, "pFFT projection left a filament's stencil box (internal error)");
    const int64_t E = out.entries;
    int32_t *d_owner, *d_lohi;
    FHB_CUDA(persist(&out.proj_idx, (size_t)E));
    FHB_CUDA(persist(&out.proj_w, (size_t)E));
    FHB_CUDA(tmp.get(&d_owner, (size_t)E));
    FHB_CUDA(tmp.get(&d_lohi, (size_t)(6 * n)));
    project_emit_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(n, g, d_boxes, d_scratch, d_touched,
                                                                    out.proj_off, out.proj_idx, out.proj_w, d_owner,
                                                                    d_lohi);
    FHB_CUDA(cudaGetLastError());
    // Transpose: stable sort of the entries by grid point.
    uint32_t *d_keys_out, *d_pos, *d_pos_out;
    FHB_CUDA(tmp.get(&d_keys_out, (size_t)E));
    FHB_CUDA(tmp.get(&d_pos, (size_t)E));
    FHB_CUDA(tmp.get(&d_pos_out, (size_t)E));
    iota_kernel<<<blocks(E, 256), 256, 0, s>>>(d_pos, E);
    FHB_CUDA(cudaGetLastError());
    int end_bit = 1;
    while (end_bit < 32 && ((int64_t)1 << end_bit) < G) ++end_bit;
    size_t sb = 0;
    FHB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sb, out.proj_idx, d_keys_out, d_pos, d_pos_out, (int)E, 0,
                                             end_bit, s));
    void *d_sb;
    FHB_CUDA(tmp.get((uint8_t **)&d_sb, sb));
    FHB_CUDA(cub::DeviceRadixSort::SortPairs(d_sb, sb, out.proj_idx, d_keys_out, d_pos, d_pos_out, (int)E, 0, end_bit,
                                             s));
    FHB_CUDA(persist(&out.spread_fil, (size_t)E));
    FHB_CUDA(persist(&out.spread_w, (size_t)E));
    gather_spread_kernel<<<blocks(E, 256), 256, 0, s>>>(d_pos_out, d_owner, out.proj_w, E, out.spread_fil,
                                                        out.spread_w);
    FHB_CUDA(cudaGetLastError());
    unsigned long long *d_gcount;
    FHB_CUDA(tmp.get(&d_gcount, (size_t)G + 1));
    FHB_CUDA(cudaMemsetAsync(d_gcount, 0, 8 * ((size_t)G + 1), s));
    count_keys_kernel<<<blocks(E, 256), 256, 0, s>>>(out.proj_idx, E, d_gcount);
    FHB_CUDA(cudaGetLastError());
    FHB_CUDA(persist(&out.spread_off, (size_t)G + 1));
    size_t tg = 0;
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tg, reinterpret_cast<int64_t *>(d_gcount), out.spread_off,
                                           (int)(G + 1), s));
    void *d_tg;
    FHB_CUDA(tmp.get((uint8_t **)&d_tg, tg));
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(d_tg, tg, reinterpret_cast<int64_t *>(d_gcount), out.spread_off,
                                           (int)(G + 1), s));
    // Grid approximations of the near pairs.
    const int64_t np = near.count;
    FHB_CUDA(persist(&out.pair_grid, (size_t)np));
    if (np) {
        const int2 *d_pairs = near.pairs;
        const int64_t *d_poff = near.off;
        int *d_reach;
        FHB_CUDA(tmp.get(&d_reach, 4));
        FHB_CUDA(cudaMemsetAsync(d_reach, 0, 16, s));
        reach_kernel<<<blocks(np, 256), 256, 0, s>>>(d_pairs, np, d_lohi, d_reach);
        FHB_CUDA(cudaGetLastError());
        int reach[4] = {0, 0, 0, 0};
        FHB_CUDA(cudaMemcpyAsync(reach, d_reach, 16, cudaMemcpyDeviceToHost, s));
        FHB_CUDA(cudaStreamSynchronize(s));
        const int64_t tsize = (int64_t)(2 * reach[0] + 1) * (2 * reach[1] + 1) * (2 * reach[2] + 1);
        double *d_table;
        FHB_CUDA(tmp.get(&d_table, (size_t)tsize));
        kernel_table_kernel<<<blocks(tsize, 256), 256, 0, s>>>(d_table, reach[0], reach[1], reach[2], g.spacing);
        FHB_CUDA(cudaGetLastError());
        const unsigned rows = (unsigned)std::min<int64_t>(n, 148 * 16);
        precorrect_kernel<<<rows, kPreThreads, 0, s>>>(n, g, d_poff, d_pairs, out.proj_off, out.proj_idx, out.proj_w,
                                                       d_table, reach[0], reach[1], reach[2], out.pair_grid);
        FHB_CUDA(cudaGetLastError());
    }
    FHB_CUDA(cudaStreamSynchronize(s));
    return FH_OK;
}

fh_status pfft_near_csr(int64_t n, int64_t np, const int2 *d_pairs, const double *d_exact, const double *d_grid,
                        const double *d_cos, cudaStream_t s, int64_t **near_off, uint32_t **near_col,
                        double **near_val, int64_t *near_entries, fh_error_info *err) {
    Scratch tmp{s, {}};
    unsigned long long *d_keys, *d_keys2, *d_rows;
    double *d_vals, *d_vals2;
    FHB_CUDA(tmp.get(&d_keys, (size_t)(2 * np)));
    FHB_CUDA(tmp.get(&d_keys2, (size_t)(2 * np)));
    FHB_CUDA(tmp.get(&d_vals, (size_t)(2 * np)));
    FHB_CUDA(tmp.get(&d_vals2, (size_t)(2 * np)));
    FHB_CUDA(tmp.get(&d_rows, (size_t)n + 1));
    FHB_CUDA(cudaMemsetAsync(d_rows, 0, 8 * ((size_t)n + 1), s));
    if (np) {
        near_entries_kernel<<<blocks(np, 256), 256, 0, s>>>(d_pairs, np, n, d_exact, d_cos, d_grid, d_keys, d_vals,
                                                            d_rows);
        FHB_CUDA(cudaGetLastError());
    }
    FHB_CUDA(persist(near_off, (size_t)n + 1));
    size_t tb = 0;
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, reinterpret_cast<int64_t *>(d_rows), *near_off, (int)(n + 1),
                                           s));
    void *d_tb;
    FHB_CUDA(tmp.get((uint8_t **)&d_tb, tb));
    FHB_CUDA(cub::DeviceScan::ExclusiveSum(d_tb, tb, reinterpret_cast<int64_t *>(d_rows), *near_off, (int)(n + 1), s));
    int64_t total = 0;
    FHB_CUDA(cudaMemcpyAsync(&total, *near_off + n, 8, cudaMemcpyDeviceToHost, s));
    if (np) {
        size_t sb = 0;
        FHB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sb, d_keys, d_keys2, d_vals, d_vals2, (int)(2 * np), 0, 64,
                                                 s));
        void *d_sb;
        FHB_CUDA(tmp.get((uint8_t **)&d_sb, sb));
        FHB_CUDA(cub::DeviceRadixSort::SortPairs(d_sb, sb, d_keys, d_keys2, d_vals, d_vals2, (int)(2 * np), 0, 64, s));
    }
    FHB_CUDA(cudaStreamSynchronize(s));
    FHB_CUDA(persist(near_col, (size_t)total));
    FHB_CUDA(persist(near_val, (size_t)total));
    if (total) {
        near_split_kernel<<<blocks(total, 256), 256, 0, s>>>(d_keys2, d_vals2, total, n, *near_col, *near_val);
        FHB_CUDA(cudaGetLastError());
    }
    FHB_CUDA(cudaStreamSynchronize(s));
    *near_entries = total;
    return FH_OK;
}

}  // namespace fhb
