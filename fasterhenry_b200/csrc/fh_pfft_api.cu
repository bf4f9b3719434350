// C ABI of the precorrected-FFT operator (fh_pfft_*): host buffers in and
// out, the operator and its device buffers behind an opaque handle.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>

#include "fh_device.cuh"
#include "fh_pfft.h"

using namespace fhb;

struct fh_pfft {
    PfftDevice dev;
    double *d_x = nullptr, *d_y = nullptr;
    size_t cap = 0;  // vectors the x / y buffers hold
    ~fh_pfft() {
        if (d_x) cudaFree(d_x);
        if (d_y) cudaFree(d_y);
    }
};

namespace {

fh_status to_config(const fh_pfft_params *p, PfftConfig &cfg, fh_error_info *err) {
    fh_pfft_params d;
    fh_pfft_default_params(&d);
    if (!p) p = &d;
    if (p->spacing_kind != 0 && p->spacing_kind != 1)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "spacing_kind must be 0 (auto) or 1 (fixed)");
    cfg.fixed_spacing = p->spacing_kind == 1;
    cfg.cells_per_filament = p->cells_per_filament;
    cfg.spacing = p->spacing;
    cfg.near_field_radius = p->near_field_radius;
    cfg.order = p->interpolation_order;
    if (p->fft_precision != 0 && p->fft_precision != 1)
        return fail(err, FH_ERR_INVALID_ARGUMENT, "fft_precision must be 0 (FP64) or 1 (FP32)");
    cfg.fft_fp32 = p->fft_precision == 1;
    return FH_OK;
}

}  // namespace

extern "C" {

void fh_pfft_default_params(fh_pfft_params *params) {
    if (!params) return;
    params->spacing_kind = 0;
    params->interpolation_order = 5;
    params->cells_per_filament = 8.0;
    params->spacing = 0.0;
    params->near_field_radius = 8.0;
    params->fft_precision = 0;
    params->reserved = 0;
}

fh_status fh_pfft_create(const fh_filament *filaments, size_t n, const fh_pfft_params *params, fh_pfft **out,
                         fh_error_info *err) {
    clear_error(err);
    if (!out || (n && !filaments)) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    PfftConfig cfg;
    fh_status st = to_config(params, cfg, err);
    if (st) return st;
    st = ensure_device(err);
    if (st) return st;
    std::unique_ptr<fh_pfft> op(new fh_pfft());
    st = pfft_build(filaments, (int64_t)n, cfg, nullptr, op->dev, err);
    if (st) return st;
    *out = op.release();
    return FH_OK;
}

fh_status fh_pfft_apply(fh_pfft *op, const double *x, double *y, size_t count, fh_error_info *err) {
    clear_error(err);
    if (!op || (op->dev.n && count && (!x || !y))) return fail(err, FH_ERR_INVALID_ARGUMENT, "null argument");
    const int64_t n = op->dev.n;
    if (n == 0 || count == 0) return FH_OK;
    if (count > 64) return fail(err, FH_ERR_INVALID_ARGUMENT, "at most 64 vectors per product");
    cudaStream_t s = (cudaStream_t)op->dev.stream;
    if (op->cap < count) {
        if (op->d_x) cudaFree(op->d_x);
        if (op->d_y) cudaFree(op->d_y);
        op->d_x = op->d_y = nullptr;
        op->cap = 0;
        if (cudaMalloc(&op->d_x, sizeof(double) * n * count) != cudaSuccess ||
            cudaMalloc(&op->d_y, sizeof(double) * n * count) != cudaSuccess) {
            cudaGetLastError();
            return fail(err, FH_ERR_OUT_OF_MEMORY, "device allocation of the product vectors failed");
        }
        op->cap = count;
    }
    FHB_CUDA(cudaMemcpyAsync(op->d_x, x, sizeof(double) * n * count, cudaMemcpyHostToDevice, s));
    fh_status st = pfft_apply(op->dev, op->d_x, op->d_y, (int)count, err);
    if (st) return st;
    FHB_CUDA(cudaMemcpyAsync(y, op->d_y, sizeof(double) * n * count, cudaMemcpyDeviceToHost, s));
    FHB_CUDA(cudaStreamSynchronize(s));
    return FH_OK;
}

fh_status fh_pfft_get_stats(const fh_pfft *op, fh_pfft_stats *stats) {
    if (!op || !stats) return FH_ERR_INVALID_ARGUMENT;
    const PfftDevice &d = op->dev;
    stats->filaments = d.n;
    stats->grid_spacing = d.grid.spacing;
    for (int a = 0; a < 3; ++a) {
        stats->grid_dims[a] = d.grid.dims[a];
        stats->fft_dims[a] = d.padded[a];
    }
    stats->projection_entries = d.projection_entries;
    stats->near_entries = d.near_entries;
    stats->memory_bytes = (int64_t)d.memory_bytes();
    stats->setup_host_s = d.setup_host_s;
    stats->setup_device_s = d.setup_device_s;
    stats->setup_near_s = d.setup_near_s;
    return FH_OK;
}

void fh_pfft_destroy(fh_pfft *op) { delete op; }

}  // extern "C"
