// Interface of the tangent-linear and adjoint kernels (adjoint.cu).
#pragma once
#include <cstdint>

#include "opgpu_device.h"

namespace opgpu {

constexpr int KAdjList = 16;                                // list capacity of the TLM / adjoint kernels
constexpr int KAdjPairs = KAdjList * (KAdjList - 1) / 2;

struct AdjArrays {
    // adjoint step: the state after the step (its lists and the adjoint of its values)
    const uint8_t* cnt1;
    const int16_t* idx1;
    const double* lam1;         // [K][N]
    double* lam_local;          // [K][N] the voxel's own part of the adjoint of the input values
    uint8_t* lcnt;              // [N]  list length of the voxel's step (0 for bulk voxels)
    int16_t* lidx;              // [KAdjList][N] grains of the list
    double* llam;               // [KAdjList][N] adjoint of the list's Laplacians
    double* gsig;               // [G*G] dL/dsigma(a,b), accumulated at a*G+b with a < b
    double* gmu;                // [G*G] dL/dmu(a,b), same layout
    double* gdg;                // [G]   dL/ddG(g)
    // tangent step
    const double* tsig;         // [G*G] tangent of sigma(a,b) at a*G+b with a < b (or null)
    const double* tmu;          // [G*G] tangent of mu(a,b) (or null)
    const double* tdg;          // [G]   tangent of dG (or null)
    const double* dphi_in;      // [K][N] tangent of the input values
    double* dphi_out;           // [K][N] tangent of the output values
    double* tvol;               // [G] tangent of the output grain volumes (accumulated)
};

// One FP64 step with tangents (writes the new state like the step kernels, and its tangent).
int launch_tlm_step(const StepParams& p, const StepArrays& a, const AdjArrays& aa, int k_slots, void* stream);
// Adjoint of one step: a.cnt_in/idx_in/val_in hold the state before the step, aa the state after it
// and its adjoint; the classify kernel has just run on the state before the step (its work
// records, buckets and worklist in a; nblocks its block count).  Writes the adjoint of the state
// before the step to lam0 and accumulates the parameter gradients.
// A side stream with a fork and a join event (cudaEvent_t, timing disabled) for the worklist
// kernel; side == nullptr runs everything on the main stream.
struct AdjStreams {
    void* side;
    void* ev_fork;
    void* ev_join;
};
int launch_adjoint_step(const StepParams& p, const StepArrays& a, const AdjArrays& aa, int k_slots, bool fp32,
                        int nblocks, double* lam0, void* stream, const AdjStreams& fork);
// lam[s][v] = dLdV[idx[s][v]] on the stored entries (adjoint of a loss on the grain volumes).
int launch_lambda_init(long long n, const uint8_t* cnt, const int16_t* idx, const double* dLdV, double* lam,
                       void* stream);

}  // namespace opgpu
