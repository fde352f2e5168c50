// K2: plaquette, clover energy and clover topological charge
// (src/Observables/superobs.cpp:31-128), one thread per (site, plane).
//
// Per plane (mu < nu) the four clover leaves, all oriented the same way,
//   Q1 = U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
//   Q2 = U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu)
//   Q3 = U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_nu(x-nu)
//   Q4 = U_nu(x-nu)^+ U_mu(x-nu) U_nu(x+mu-nu) U_mu(x)^+
// give C = sum Q and G = [C - C^+]_traceless.  The reference adds Q1 and Q3 and
// subtracts Q4^+ and Q2^+ (superobs.cpp:47-74); after C - C^+ both sums give the
// same G.  Per site:
//   plaq   += Re tr Q1                        (:71, normalised by 18 V at :125)
//   energy += Re tr(G_{mu nu} G_{mu nu})      (:109, raw, no 1/8 factor)
//   topc   -= Re tr(G01 G23) + Re tr(G02 G13^+) + Re tr(G03 G12)   (:114-124, / 256 pi^2)
// Planes are visited in the pairs (01,23), (02,13), (03,12) so only two G are
// live at a time.  Site values are accumulated in FP64 whatever the link
// precision: warp shuffles, a shared-memory tree, one partial per block, and a
// single-block fold in a fixed order (deterministic, no atomics), in place of
// the reference's MPI_Allreduce (:24-28).
#include "kernels.h"
#include "observables.cuh"

namespace ym {

// One block of 1024 threads: thread i folds partials i, i+1024, ... in order,
// then the block tree.  Output (plaq, topc, energy, nonfinite flag).
__global__ void __launch_bounds__(1024) obs_finalize_kernel(const double* partials, int nblocks, double inv_18v,
                                                            double* out) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
        a += partials[3 * i + 0];
        b += partials[3 * i + 1];
        c += partials[3 * i + 2];
    }
    block_sum3(a, b, c);
    if (threadIdx.x == 0) {
        const double plaq = a * inv_18v;
        const double topc = c / (256.0 * 3.14159265358979323846 * 3.14159265358979323846);
        out[0] = plaq;
        out[1] = topc;
        out[2] = b;
        out[3] = (isfinite(plaq) && isfinite(topc) && isfinite(b)) ? 0.0 : 1.0;
    }
}

int obs_blocks(const Geo& g) {
    const int groups = (g.site1 - g.site0 + kObsSites - 1) / kObsSites;
    return groups < kObsMaxBlocks ? groups : kObsMaxBlocks;
}

cudaError_t launch_observables(int prec, const void* u, const Geo& g, double* partials, cudaStream_t st) {
    const unsigned nb = unsigned(obs_blocks(g));
    if (nb == 0) return cudaErrorInvalidValue;
    switch (prec) {
        case kFP64:
            observables_kernel<<<nb, kObsThreads, 0, st>>>(FieldD18{const_cast<void*>(u), g.V}, g, partials);
            break;
        case kFP32_18:
            observables_kernel<<<nb, kObsThreads, 0, st>>>(FieldF18{const_cast<void*>(u), g.V}, g, partials);
            break;
        case kFP32_12:
            observables_kernel<<<nb, kObsThreads, 0, st>>>(FieldF12{const_cast<void*>(u), g.V}, g, partials);
            break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_obs_finalize(const double* partials, int nblocks, const Geo& g, double* out, cudaStream_t st) {
    obs_finalize_kernel<<<1, 1024, 0, st>>>(partials, nblocks, 1.0 / (18.0 * double(g.vglobal)), out);
    return cudaGetLastError();
}

}  // namespace ym
