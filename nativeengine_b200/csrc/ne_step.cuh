// ne_step.cuh -- by-value launch arguments of the step kernels.
#pragma once

#include "ne_internal.cuh"

namespace neb {

struct StepArgs {
    DevWorld d;
    uint32_t n;              // bodies
    Domain dom;              // Box (half, periodic)
    double dt, restitution, friction, beta;
    V3 g;                    // gravity
    int rcomb, fcomb;        // material combine modes
    int warm;                // World::warmStart
    int open_boundary;
    // broadphase constants (fixed per upload: cell = 2 * max bounding radius)
    double cell;
    long long nc[3];
    int brute;               // forceBruteForce || n < 64 || cell < 1e-9
    uint32_t nplanes;
    int key_bits;            // bits the cell-key sort covers this step
    // capacities
    uint64_t Pcap, Scap, Ccap;
    int num_sms;
};

// ev: NE_NUM_STAGES + 1 events recorded at the stage boundaries, or nullptr.
void launch_step(const StepArgs& a, cudaStream_t st, uint64_t* launches, cudaEvent_t* ev);

}  // namespace neb
