// hhg_noalloc.cu -- the allocation-free entry point hhg_gpu_current_density_noalloc
// and its status query hhg_noalloc_status.
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
// share the array and it keeps the last call's contents; a set-up kernel
// clears the counters and rewrites the pulse record and time grid on every
// call, and every other byte the kernels read is written by the staging
// kernel first.  Calls whose work overlaps on the GPU (different streams, or
// different host threads on one device) race on the array and must be
// serialised by the caller.
//
// The call enqueues kernels only (the pulse record travels as a kernel
// argument, the time grid is accumulated on the device), so no copy reads
// host memory after the call returns.  The scratch address is looked up once
// per device and cached; this assumes the device's primary context for the
// life of the process (after cudaDeviceReset the module, and the array, may
// be reloaded at another address).
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
// Under stream capture only a cached address is used: the first lookup may
// load the module, which a capture must not see.
hhg_status scratch_for_device(int dev, unsigned char **out, char *err, size_t cap,
                              bool capturing = false) {
    if (dev < 0 || dev >= kMaxDevices) {
        set_msg(err, cap, "device ordinal out of range for the scratch table");
        return HHG_BAD_CONFIG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev] && capturing) {
        set_msg(err, cap, "the first allocation-free call on a device must come before any stream capture");
        return HHG_UNSUPPORTED;
    }
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

// Whether `s` is being captured into a graph (an error querying it counts as
// capturing: the caller then takes the capture-safe path or refuses).
bool stream_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
        (void)cudaGetLastError();
        return true;
    }
    return cs != cudaStreamCaptureStatusNone;
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

// Scratch header (first 256 bytes): the kernels' counters [0] next item,
// [1] attempted, [2] rejected, [3] failed, [4] non-finite (unsigned long
// long), the status word at byte 64, and the last call's k rows, degree and
// work items for hhg_noalloc_status.
constexpr size_t kOffStatus = 64;
constexpr size_t kOffInfo = 128;
struct NoAllocInfo {
    long long n_rows;
    long long items;
    int degree;
    int pad;
};

// One thread: clears the counters and the status word, records the call's
// sizes, writes the pulse record and the interval offsets, and accumulates the
// measurement times exactly as the host does (t_end += measure_every, a serial
// sum of doubles, so the grid is bitwise the regular entry point's).
__global__ void noalloc_setup_kernel(hhg::PulseDev pd, long long n_meas, NoAllocInfo info,
                                     unsigned char *base, hhg::PulseDev *d_pulse,
                                     long long *d_ioff, double *d_tgrid) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(base);
    for (int c = 0; c < 8; ++c) cnt[c] = 0ull;
    *reinterpret_cast<int *>(base + kOffStatus) = 0;
    *reinterpret_cast<NoAllocInfo *>(base + kOffInfo) = info;
    *d_pulse = pd;
    d_ioff[0] = 0;
    d_ioff[1] = n_meas;
    double t_begin = pd.window_begin, t_end = t_begin + pd.measure_every;
    d_tgrid[0] = t_begin;
    for (long long i = 1; i <= n_meas; ++i) {
        d_tgrid[i] = t_end;
        t_begin = t_end;
        t_end += pd.measure_every;
    }
}

// Counters and status word of the last call on the current device -> stats
// and the status code (synchronises the stream).
hhg_status read_outcome(unsigned char *base, cudaStream_t s, hhg_stats *stats, char *err,
                        size_t err_cap) {
    unsigned long long cnt[8];
    int status_h = 0;
    NoAllocInfo info{};
    cudaError_t e;
    if ((e = cudaMemcpyAsync(cnt, base, sizeof cnt, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&status_h, base + kOffStatus, sizeof status_h, cudaMemcpyDeviceToHost,
                             s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&info, base + kOffInfo, sizeof info, cudaMemcpyDeviceToHost, s)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        set_msg(err, err_cap, cudaGetErrorString(e));
        return HHG_CUDA_ERROR;
    }
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->k_points = info.n_rows;
        stats->trajectories = info.n_rows;
        stats->attempted_steps = (int64_t)cnt[1];
        stats->rejected_steps = (int64_t)cnt[2];
        stats->failed_trajectories = (int64_t)(cnt[3] + cnt[4]);
        stats->poly_degree = info.degree;
        stats->items = (int32_t)info.items;
    }
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
        (o.stepper == HHG_STEPPER_MAGNUS4 &&
         (o.precision != HHG_PREC_FP64 || !hhg_prep::magnus_substeps_ok(o.magnus_substeps))) ||
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
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool capturing = stream_capturing(s);
    if (capturing && stats) {
        set_msg(err, err_cap, "stats != NULL synchronises the stream: pass NULL under stream capture "
                              "and read the outcome with hhg_noalloc_status after the replay");
        return HHG_UNSUPPORTED;
    }
    unsigned char *base = nullptr;
    if ((st = scratch_for_device(dev, &base, err, err_cap, capturing)) != HHG_OK) return st;

    hhg::PulseDev pd = prep.pulse;
    pd.coef_off = 0;
    pd.part_off = 0;
    pd.j_off = 0;
    pd.items = (int)items;
    unsigned long long *counters = reinterpret_cast<unsigned long long *>(base);
    int *status = reinterpret_cast<int *>(base + kOffStatus);
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
    const NoAllocInfo info{(long long)n_rows, items, prep.degree, 0};
    noalloc_setup_kernel<<<1, 32, 0, s>>>(pd, (long long)N, info, base, d_pulse, d_ioff, d_tgrid);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);

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
    lr.kp.coarsen = 1.0 / hhg::kCoarsenDivFp64;  // dyadic stepping only; not offered here
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
    return read_outcome(base, s, stats, err, err_cap);
}

extern "C" hhg_status hhg_noalloc_status(void *stream, hhg_stats *stats, char *err, size_t err_cap) {
    set_msg(err, err_cap, "");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_msg(err, err_cap, "no current CUDA device");
        return HHG_CUDA_ERROR;
    }
    if (stream_capturing(static_cast<cudaStream_t>(stream))) {
        set_msg(err, err_cap, "hhg_noalloc_status synchronises the stream: not under stream capture");
        return HHG_UNSUPPORTED;
    }
    unsigned char *base = nullptr;
    const hhg_status st = scratch_for_device(dev, &base, err, err_cap);
    if (st != HHG_OK) return st;
    return read_outcome(base, static_cast<cudaStream_t>(stream), stats, err, err_cap);
}
