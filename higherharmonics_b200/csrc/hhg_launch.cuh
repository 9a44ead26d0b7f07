// hhg_launch.cuh -- per-model kernel instantiation and launch dispatch.  Each
// kernels_<model>.cu includes this header once with HHG_MODEL set, so the
// model families compile in parallel translation units.
#pragma once

#include "hhg_device.cuh"

namespace hhg {

struct LaunchReq {
    KParams kp;
    int degree;     // 5, 7 or 11; 0 = exact pulse evaluation (FP64 RKF78, proposer 0/1)
    int precision;  // 0 FP64, 1 mixed (FP32 right-hand side)
    int stepper;    // 0 RKF78, 1 Magnus-4
    int proposer;   // 0 restart at dt0, 1 carry, 2 warp-synchronous dyadic, 3 learned dyadic,
                    // 4 carry + history recording
    int grid;       // CTAs; 0 = query occupancy only
    cudaStream_t stream;
    int *occupancy_out;  // blocks per SM for the selected variant (if non-null)
    int out_mode = 0;    // bz_integrate_kernel's OUT (1-3: PiFlux models, FP64, proposer 0/1;
                         // 4: Dirac-3D models, FP64, proposer 0)
};

struct StageReq {
    const PulseDev *pulses;
    int n_pulses;
    const double *tgrid;
    const long long *interval_off;
    double *coef;
    long long total_intervals;
    int degree;
    double grow_max;
    cudaStream_t stream;
    int layout = 0;  // 0 standard schedule, 1 dyadic FP64, 2 dyadic float pairs, 3 Dirac Magnus moments
    const double *gl30 = nullptr;  // layout 3: 30 nodes on [0, 1], then 30 weights (device)
};

template <int M, int D, typename R, int ST, int PR, int OUT = 0>
cudaError_t launch_one(const LaunchReq &r) {
    auto kern = bz_integrate_kernel<M, D, R, ST, PR, OUT>;
    const int dyn = PR == 3 ? mlp_smem_bytes() : 0;
    if (r.occupancy_out) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(r.occupancy_out, kern, kBlockThreads, dyn);
        if (e != cudaSuccess) return e;
    }
    if (r.grid <= 0) return cudaSuccess;
    kern<<<r.grid, kBlockThreads, dyn, r.stream>>>(r.kp);
    return cudaGetLastError();
}

// k-resolved and split-current outputs (OUT 1-3): PiFlux models, FP64 RKF78,
// the reference schedule or the carried step.  Per-trajectory current (OUT
// 4): the Dirac-3D models, FP64, the reference schedule or (coherent) the
// closed-form Magnus step.
template <int M, int D>
cudaError_t launch_out(const LaunchReq &r) {
    if constexpr (base_model(M) == DIRAC3D) {
        if (r.out_mode != 4 || r.precision != 0 || r.proposer != 0) return cudaErrorNotSupported;
        if (r.stepper == 0) return launch_one<M, D, double, 0, 0, 4>(r);
        if constexpr (M == DIRAC3D) {
            if (r.stepper == 2) return launch_one<M, D, double, 2, 0, 4>(r);
        }
        return cudaErrorNotSupported;
    } else if constexpr (base_model(M) == PIFLUX3D) {
        if (r.stepper != 0 || r.precision != 0 || (r.proposer != 0 && r.proposer != 1))
            return cudaErrorNotSupported;
        const bool carry = r.proposer == 1;
        switch (r.out_mode) {
        case 1: return carry ? launch_one<M, D, double, 0, 1, 1>(r) : launch_one<M, D, double, 0, 0, 1>(r);
        case 2: return carry ? launch_one<M, D, double, 0, 1, 2>(r) : launch_one<M, D, double, 0, 0, 2>(r);
        case 3: return carry ? launch_one<M, D, double, 0, 1, 3>(r) : launch_one<M, D, double, 0, 0, 3>(r);
        }
        return cudaErrorInvalidValue;
    } else {
        return cudaErrorNotSupported;
    }
}

template <int M, int D>
cudaError_t launch_deg(const LaunchReq &r) {
    if (r.out_mode != 0) return launch_out<M, D>(r);
    if constexpr (Traits<M>::kRelax) {
        // relaxation right-hand sides: FP64 controlled RKF78 only
        if (r.stepper != 0 || r.precision != 0) return cudaErrorNotSupported;
        switch (r.proposer) {
        case 0: return launch_one<M, D, double, 0, 0>(r);
        case 1: return launch_one<M, D, double, 0, 1>(r);
        case 2: return launch_one<M, D, double, 0, 2>(r);
        case 3: return launch_one<M, D, double, 0, 3>(r);
        case 4: return launch_one<M, D, double, 0, 4>(r);
        }
        return cudaErrorInvalidValue;
    } else {
        if (r.stepper == 2) {
            // the reference's closed-form Dirac Magnus step
            if constexpr (M == DIRAC3D) return launch_one<M, D, double, 2, 0>(r);
            else return cudaErrorNotSupported;
        }
        if (r.stepper == 1) return launch_one<M, D, double, 1, 0>(r);
        if (r.precision == 0) {
            switch (r.proposer) {
            case 0: return launch_one<M, D, double, 0, 0>(r);
            case 1: return launch_one<M, D, double, 0, 1>(r);
            case 2: return launch_one<M, D, double, 0, 2>(r);
            case 3: return launch_one<M, D, double, 0, 3>(r);
            case 4: return launch_one<M, D, double, 0, 4>(r);
            }
            return cudaErrorInvalidValue;
        }
        switch (r.proposer) {
        case 0: return launch_one<M, D, float, 0, 0>(r);
        case 1: return launch_one<M, D, float, 0, 1>(r);
        case 2: return launch_one<M, D, float, 0, 2>(r);
        case 3: return launch_one<M, D, float, 0, 3>(r);
        }
        return cudaErrorInvalidValue;
    }
}

// Degree 0 (pulses evaluated exactly at every stage time, no interpolant):
// FP64 RKF78 with the reference schedule or the carried step, the current
// only.
template <int M>
cudaError_t launch_exact(const LaunchReq &r) {
    if (r.out_mode != 0 || r.stepper != 0 || r.precision != 0) return cudaErrorNotSupported;
    if (r.proposer == 0) return launch_one<M, 0, double, 0, 0>(r);
    if (r.proposer == 1) return launch_one<M, 0, double, 0, 1>(r);
    return cudaErrorNotSupported;
}

template <int M>
cudaError_t launch_model(const LaunchReq &r) {
    if (r.degree == 0) return launch_exact<M>(r);
    if (r.degree == 5) return launch_deg<M, 5>(r);
    if (r.degree == 7) return launch_deg<M, 7>(r);
    if (r.degree == 11) return launch_deg<M, 11>(r);
    return cudaErrorInvalidValue;
}

template <int M, int D, int LAYOUT>
void stage_one(const StageReq &s, unsigned blocks, int threads) {
    stage_pulses_kernel<M, D, LAYOUT><<<blocks, threads, 0, s.stream>>>(
        s.pulses, s.n_pulses, s.tgrid, s.interval_off, s.coef, s.total_intervals, s.grow_max,
        s.gl30);
}

template <int M, int D>
void stage_deg(const StageReq &s, unsigned blocks, int threads) {
    if (s.layout == 0) stage_one<M, D, 0>(s, blocks, threads);
    else if (s.layout == 1) stage_one<M, D, 1>(s, blocks, threads);
    else if (s.layout == 2) stage_one<M, D, 2>(s, blocks, threads);
    else if constexpr (M == DIRAC3D) stage_one<M, D, 3>(s, blocks, threads);
}

template <int M>
cudaError_t stage_model(const StageReq &s) {
    const int threads = 128;
    const long long blocks = (s.total_intervals + threads - 1) / threads;
    if (s.layout < 0 || s.layout > 3 || (s.layout == 3 && (M != DIRAC3D || !s.gl30)))
        return cudaErrorInvalidValue;
    if (s.degree == 0) {
        if (s.layout != 0) return cudaErrorNotSupported;
        stage_one<M, 0, 0>(s, (unsigned)blocks, threads);
    } else if (s.degree == 5) stage_deg<M, 5>(s, (unsigned)blocks, threads);
    else if (s.degree == 7) stage_deg<M, 7>(s, (unsigned)blocks, threads);
    else if (s.degree == 11) stage_deg<M, 11>(s, (unsigned)blocks, threads);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_dirac2d(const LaunchReq &r);
cudaError_t launch_piflux2d(const LaunchReq &r);
cudaError_t launch_piflux3d(const LaunchReq &r);
cudaError_t launch_honeycomb(const LaunchReq &r);
cudaError_t launch_dirac3d(const LaunchReq &r);
cudaError_t launch_piflux2d_sym(const LaunchReq &r);
cudaError_t launch_honeycomb_x(const LaunchReq &r);
cudaError_t launch_piflux3d_relax(const LaunchReq &r);
cudaError_t launch_honeycomb_relax(const LaunchReq &r);
cudaError_t launch_dirac3d_relax(const LaunchReq &r);
cudaError_t stage_dirac2d(const StageReq &s);
cudaError_t stage_piflux2d(const StageReq &s);
cudaError_t stage_piflux3d(const StageReq &s);
cudaError_t stage_honeycomb(const StageReq &s);
cudaError_t stage_dirac3d(const StageReq &s);
cudaError_t stage_piflux2d_sym(const StageReq &s);
cudaError_t stage_honeycomb_x(const StageReq &s);
cudaError_t stage_piflux3d_relax(const StageReq &s);
cudaError_t stage_honeycomb_relax(const StageReq &s);
cudaError_t stage_dirac3d_relax(const StageReq &s);

}  // namespace hhg

#ifdef HHG_MODEL
#define HHG_CAT2(a, b) a##b
#define HHG_CAT(a, b) HHG_CAT2(a, b)
namespace hhg {
cudaError_t HHG_CAT(launch_, HHG_MODEL_NAME)(const LaunchReq &r) { return launch_model<HHG_MODEL>(r); }
cudaError_t HHG_CAT(stage_, HHG_MODEL_NAME)(const StageReq &s) { return stage_model<HHG_MODEL>(s); }
}  // namespace hhg
#endif
