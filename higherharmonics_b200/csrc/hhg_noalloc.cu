// hhg_noalloc.cu -- the allocation-free entry point hhg_gpu_current_density_noalloc.
//
// Some callers cannot allocate device memory while they call this library:
// code running inside another framework's memory pool or allocator hooks,
// real-time loops that must not call cudaMalloc (it can synchronise the
// device and take milliseconds), and processes that pre-plan every byte of a
// GPU shared with other jobs.  For them the integration kernel's scratch --
// the per-interval pulse staging, the per-work-item partial current rows and
// the work/status counters -- lives in the file-scope device array below.
// The caller passes the inputs (the k table in device memory) and the output
// (j in device memory); nothing here calls cudaMalloc, cudaFree or a library
// routine that allocates.
//
// The array is part of this module: every GPU that loads it (its first use on
// that device) holds kNoAllocScratchBytes until the process exits.  All calls
// share the array and it keeps the last call's contents; the counters are
// cleared on every call and every other byte the kernels read is rewritten
// first.  Calls whose work overlaps on the GPU (different streams, or
// different host threads on one device) race on the array and must be
// serialised by the caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/hhg_gpu.h"
#include "hhg_launch.cuh"
#include "hhg_pulse_prep.hpp"

namespace {

// 64 MiB: e.g. a 128x128 grid over 8192 intervals for any model family.
constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_ptr[kMaxDevices] = {};

size_t round256(size_t n) { return (n + 255) & ~size_t(255); }

void set_msg(char *buf, size_t cap, const char *msg) {
    if (buf && cap) {
        std::strncpy(buf, msg, cap - 1);
        buf[cap - 1] = '\0';
    }
}

// Device address of the scratch array on the current device.  In host code
// the name g_noalloc_scratch is only a host-side stand-in, so the address is
// looked up once per device (with that device current) and cached.
hhg_status scratch_for_device(int dev, unsigned char **out, char *err, size_t cap) {
    if (dev < 0 || dev >= kMaxDevices) {
        set_msg(err, cap, "device ordinal out of range for the scratch table");
        return HHG_BAD_CONFIG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_msg(err, cap, cudaGetErrorString(e));
            return HHG_CUDA_ERROR;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_ptr[dev]);
    return HHG_OK;
}

cudaError_t launch_model(int model, const hhg::LaunchReq &r) {
    switch (model) {
    case hhg::DIRAC2D: return hhg::launch_dirac2d(r);
    case hhg::PIFLUX2D: return hhg::launch_piflux2d(r);
    case hhg::PIFLUX3D: return hhg::launch_piflux3d(r);
    case hhg::HONEYCOMB: return hhg::launch_honeycomb(r);
    case hhg::DIRAC3D: return hhg::launch_dirac3d(r);
    case hhg::PIFLUX2D_SYM: return hhg::launch_piflux2d_sym(r);
    case hhg::HONEYCOMB_X: return hhg::launch_honeycomb_x(r);
    }
    return cudaErrorInvalidValue;
}

cudaError_t stage_model(int model, const hhg::StageReq &s) {
    switch (model) {
    case hhg::DIRAC2D: return hhg::stage_dirac2d(s);
    case hhg::PIFLUX2D: return hhg::stage_piflux2d(s);
    case hhg::PIFLUX3D: return hhg::stage_piflux3d(s);
    case hhg::HONEYCOMB: return hhg::stage_honeycomb(s);
    case hhg::DIRAC3D: return hhg::stage_dirac3d(s);
    case hhg::PIFLUX2D_SYM: return hhg::stage_piflux2d_sym(s);
    case hhg::HONEYCOMB_X: return hhg::stage_honeycomb_x(s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

extern "C" hhg_status hhg_gpu_current_density_noalloc(const hhg_system_desc *sys,
                                                      const hhg_pulse_desc *pulse,
                                                      const double *d_rows, int64_t n_rows,
                                                      const hhg_solver_opts *opts,
                                                      double *d_j_out, void *stream,
                                                      hhg_stats *stats, char *err,
                                                      size_t err_cap) {
    set_msg(err, err_cap, "");
    if (!d_rows || !d_j_out || n_rows < 1 || n_rows > (int64_t(1) << 31)) {
        set_msg(err, err_cap, "need device k rows (1 <= n_rows <= 2^31) and a device j buffer");
        return HHG_BAD_CONFIG;
    }
    hhg_solver_opts o;
    hhg_default_solver_opts(&o);
    if (opts) o = *opts;
    if (o.proposer != HHG_PROPOSER_NONE && o.proposer != HHG_PROPOSER_CARRY) {
        set_msg(err, err_cap, "the allocation-free entry point supports the restart and carry proposers");
        return HHG_UNSUPPORTED;
    }
    if ((o.stepper != HHG_STEPPER_RKF78 && o.stepper != HHG_STEPPER_MAGNUS4) ||
        (o.precision != HHG_PREC_FP64 && o.precision != HHG_PREC_MIXED) ||
        (o.stepper == HHG_STEPPER_MAGNUS4 && (o.precision != HHG_PREC_FP64 || o.magnus_substeps < 1)) ||
        !(o.abs_tol >= 0.0) || !(o.rel_tol >= 0.0) || !(o.abs_tol + o.rel_tol > 0.0)) {
        set_msg(err, err_cap, "invalid solver options");
        return HHG_BAD_CONFIG;
    }
    if (o.max_failed_steps < 1) o.max_failed_steps = 500;
    if (o.max_attempts_per_interval < 1) o.max_attempts_per_interval = 100000;

    if (pulse && pulse->kind == HHG_PULSE_SPLINE) {
        set_msg(err, err_cap, "the allocation-free entry point takes the analytic pulse shapes, not splines");
        return HHG_UNSUPPORTED;
    }
    hhg_prep::PulsePrep prep;
    hhg_status st = hhg_prep::prepare_pulse(sys, pulse, prep);
    if (st != HHG_OK) {
        set_msg(err, err_cap, "invalid system or pulse descriptor");
        return st;
    }
    if (prep.degree < 0) {
        set_msg(err, err_cap, "measurement interval too coarse for the staged pulse interpolants");
        return HHG_UNSUPPORTED;
    }
    if (sys->inv_diag_relax > 0.0) {
        set_msg(err, err_cap, "the allocation-free entry point integrates the coherent equations only");
        return HHG_UNSUPPORTED;
    }
    const int N = pulse->n_measurements;
    const int slot = hhg::slot_doubles(prep.nf, prep.degree);
    const long long items = (n_rows + 31) / 32;

    // scratch layout: [counters+status 256 B][pulse][interval offsets][tgrid][staging][partials]
    const size_t off_pulse = 256;
    const size_t off_ioff = off_pulse + round256(sizeof(hhg::PulseDev));
    const size_t off_tgrid = off_ioff + 256;
    const size_t off_coef = off_tgrid + round256(sizeof(double) * (size_t)(N + 1));
    const size_t off_part = off_coef + round256(sizeof(double) * (size_t)N * slot);
    const size_t need = off_part + sizeof(double) * (size_t)items * (size_t)(N + 1);
    if (need > kNoAllocScratchBytes) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "problem needs %zu bytes of scratch; the allocation-free entry point has %zu "
                      "(fewer k rows or measurement intervals, or use hhg_gpu_current_density)",
                      need, kNoAllocScratchBytes);
        set_msg(err, err_cap, msg);
        return HHG_BAD_CONFIG;
    }

    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        set_msg(err, err_cap, "no current CUDA device");
        return HHG_CUDA_ERROR;
    }
    unsigned char *base = nullptr;
    if ((st = scratch_for_device(dev, &base, err, err_cap)) != HHG_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    hhg::PulseDev pd = prep.pulse;
    pd.coef_off = 0;
    pd.part_off = 0;
    pd.j_off = 0;
    pd.items = (int)items;
    const long long ioff[2] = {0, N};
    unsigned long long *counters = reinterpret_cast<unsigned long long *>(base);
    int *status = reinterpret_cast<int *>(base + 64);
    hhg::PulseDev *d_pulse = reinterpret_cast<hhg::PulseDev *>(base + off_pulse);
    long long *d_ioff = reinterpret_cast<long long *>(base + off_ioff);
    double *d_tgrid = reinterpret_cast<double *>(base + off_tgrid);
    double *d_coef = reinterpret_cast<double *>(base + off_coef);
    double *d_part = reinterpret_cast<double *>(base + off_part);

    auto fail = [&](cudaError_t e) {
        set_msg(err, err_cap, cudaGetErrorString(e));
        return HHG_CUDA_ERROR;
    };
    cudaError_t e;
    // pageable sources: each copy has consumed its source when it returns
    if ((e = cudaMemsetAsync(base, 0, 256, s)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpyAsync(d_pulse, &pd, sizeof pd, cudaMemcpyHostToDevice, s)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpyAsync(d_ioff, ioff, sizeof ioff, cudaMemcpyHostToDevice, s)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpyAsync(d_tgrid, prep.tgrid.data(), sizeof(double) * (N + 1), cudaMemcpyHostToDevice, s)) != cudaSuccess) return fail(e);

    const double grow_max = 9.0 / 10.0 * pow(pow(5.0, -8.0), -1.0 / 8);
    hhg::StageReq sr{d_pulse, 1, d_tgrid, d_ioff, d_coef, (long long)N, prep.degree, grow_max, s};
    if ((e = stage_model(prep.model, sr)) != cudaSuccess) return fail(e);

    hhg::LaunchReq lr{};
    lr.kp.ktab = d_rows;
    lr.kp.pulses = d_pulse;
    lr.kp.coef = d_coef;
    lr.kp.part = d_part;
    lr.kp.counters = counters;
    lr.kp.status = status;
    lr.kp.n_items = items;
    lr.kp.n_k = (int)n_rows;
    lr.kp.tiles_per_item = 1;
    lr.kp.items_per_pulse = (int)items;
    lr.kp.max_failed = o.max_failed_steps;
    lr.kp.max_attempts = o.max_attempts_per_interval;
    lr.kp.magnus_substeps = o.magnus_substeps;
    lr.kp.abs_tol = o.abs_tol;
    lr.kp.rel_tol = o.rel_tol;
    lr.kp.err_floor = pow(5.0, -8.0);
    lr.kp.grow_max = grow_max;
    lr.degree = prep.degree;
    lr.precision = o.precision;
    lr.stepper = o.stepper;
    lr.proposer = o.proposer;
    int occ = 0;
    lr.grid = 0;
    lr.occupancy_out = &occ;
    if ((e = launch_model(prep.model, lr)) != cudaSuccess) return fail(e);
    const long long max_ctas = (long long)(occ > 0 ? occ : 1) * sms;
    const long long want = (items + hhg::kWarpsPerBlock - 1) / hhg::kWarpsPerBlock;
    lr.grid = (int)(want < max_ctas ? want : max_ctas);
    lr.occupancy_out = nullptr;
    lr.stream = s;
    if ((e = launch_model(prep.model, lr)) != cudaSuccess) return fail(e);
    hhg::reduce_partials_kernel<<<(unsigned)hhg::reduce_blocks((long long)N + 1), hhg::kReduceThreads, 0, s>>>(
        d_pulse, 1, d_part, d_j_out, (long long)N + 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);

    if (!stats) return HHG_OK;
    // counters and status word to the host (fixed-size stack copy)
    unsigned long long cnt[8];
    int status_h = 0;
    if ((e = cudaMemcpyAsync(cnt, counters, sizeof cnt, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpyAsync(&status_h, status, sizeof status_h, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return fail(e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e);
    std::memset(stats, 0, sizeof *stats);
    stats->k_points = n_rows;
    stats->trajectories = n_rows;
    stats->attempted_steps = (int64_t)cnt[1];
    stats->rejected_steps = (int64_t)cnt[2];
    stats->failed_trajectories = (int64_t)(cnt[3] + cnt[4]);
    stats->poly_degree = prep.degree;
    stats->items = (int32_t)items;
    if (status_h == 2) {
        set_msg(err, err_cap, "a trajectory exceeded the failed-step or step limit");
        return HHG_STEP_LIMIT;
    }
    if (status_h == 3) {
        set_msg(err, err_cap, "non-finite Bloch vector");
        return HHG_NONFINITE;
    }
    return HHG_OK;
}
