// Pupil sample tables in shared memory (pupil/quadrature.hpp:71 of the reference): the
// kernel parameter block carries rho_i, W_i/M with square roots and sin/cos of the azimuths;
// each CTA copies them once into shared memory for thread-dependent indexing.
#pragma once

#include "common.cuh"

namespace mkb {

// Shared pupil tables copied from the parameter block once per CTA.
struct SharedTables {
    double rho[kMaxRings];
    double w_axis[kMaxRings], rw_axis[kMaxRings];
    double w_spoke[kMaxRings], rw_spoke[kMaxRings];
    double sin_half[kMaxSpokes], cos_half[kMaxSpokes];
    double sin_full[kMaxSpokes], cos_full[kMaxSpokes];
};

__device__ inline void copy_tables(const TraceParams& p, SharedTables& t) {
    for (int i = threadIdx.x; i < kMaxRings; i += blockDim.x) {
        t.rho[i] = p.rho[i];
        t.w_axis[i] = p.w_axis[i];
        t.rw_axis[i] = p.rw_axis[i];
        t.w_spoke[i] = p.w_spoke[i];
        t.rw_spoke[i] = p.rw_spoke[i];
    }
    for (int i = threadIdx.x; i < kMaxSpokes; i += blockDim.x) {
        t.sin_half[i] = p.sin_half[i];
        t.cos_half[i] = p.cos_half[i];
        t.sin_full[i] = p.sin_full[i];
        t.cos_full[i] = p.cos_full[i];
    }
}

// Sample k of field f: rho, weight and sin/cos of the azimuth (pupil/quadrature.hpp:71).
struct Sample {
    double rho, weight, root_weight, sin_phi, cos_phi;
};

__device__ inline Sample pupil_sample(const TraceParams& p, const SharedTables& t, int f, int k) {
    Sample s;
    const int mode = p.pupil_mode[f];
    if (mode == MKB_PUPIL_AXIS) {
        s.rho = t.rho[k];
        s.weight = t.w_axis[k];
        s.root_weight = t.rw_axis[k];
        s.sin_phi = 0.0;
        s.cos_phi = 1.0;
    } else {
        const int i = k / p.spokes;
        const int j = k - i * p.spokes;
        s.rho = t.rho[i];
        s.weight = t.w_spoke[i];
        s.root_weight = t.rw_spoke[i];
        if (mode == MKB_PUPIL_HALF) {
            s.sin_phi = t.sin_half[j];
            s.cos_phi = t.cos_half[j];
        } else {
            s.sin_phi = t.sin_full[j];
            s.cos_phi = t.cos_full[j];
        }
    }
    return s;
}

}  // namespace mkb
