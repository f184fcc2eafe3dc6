/*
 * Drop-in GPU implementation of lpmCxx's Lpm::DirectSum and Lpm::TreeSum (declared by the reference's
 * own src/LpmDirectSum.h and src/LpmTreeSum.h).  Build the reference with LpmDirectSumB200.cpp and
 * LpmTreeSumB200.cpp in place of src/LpmDirectSum.cpp and src/LpmTreeSum.cpp and link liblpm_b200.so:
 * every caller keeps the reference's constructors and methods, and the pair loops run on the GPU
 * through the C ABI of include/lpm_b200.h.
 *
 * Behaviour kept from the reference: outputs written into the target Field in place (comp0/1/2), only
 * the targets of the calling rank's MPIReplicatedData ranges, divided faces untouched; an unsupported
 * kernel throws std::logic_error("invalid kernel") (src/LpmDirectSum.cpp:168-172); allocation failures
 * throw std::bad_alloc; other library failures throw std::runtime_error with lpm_last_error().  There
 * is no CPU fallback.  meshBroadcast / meshfreeBroadcast are no-ops: one GPU computes every target of
 * the calling rank, and ranks that need the other slices exchange them exactly as before by calling
 * the reference's broadcast on their own (single-GPU runs have one rank).
 *
 * Kernel mapping (lpm_kernel_desc): BiotSavartSphere(delta, R) (src/LpmVectorKernel.h:19-39) and the
 * ScalarKernel family (SphereGreensFn, PlanarGreensFnFreeBoundaries, SecondOrderDelta3d, SphereDelta;
 * src/LpmScalarKernel.h:19-78), whose parameters are recovered through their public interface, and
 * PoissonGreensFn3d below, the 3D Poisson kernel the reference lacks.  The ScalarKernel family runs in
 * FP64 only (LPM_B200_PRECISION=f32 applies to Biot-Savart and PoissonGreensFn3d).
 */
#ifndef LPM_B200_DROPIN_H
#define LPM_B200_DROPIN_H

#include "LpmScalarKernel.h"
#include "LpmTypeDefs.h"
#include "LpmVectorKernel.h"
#include "LpmXyzVector.h"

#include "lpm_b200.h"

#include <cmath>
#include <memory>
#include <string>

namespace Lpm {

/// 1/(4 pi |x - y|), zero at x == y: the scalar kernel of the 3D Poisson problem.
class PoissonGreensFn3d : public ScalarKernel {
   public:
    PoissonGreensFn3d() {}
    inline scalar_type evaluate(const XyzVector& tgtLoc, const XyzVector& srcLoc) const {
        const scalar_type r = (tgtLoc - srcLoc).magnitude();
        return r > 0.0 ? 1.0 / (4.0 * PI * r) : 0.0;
    }
    inline bool isSingular() const { return true; }
};

namespace b200 {

/// The process-wide library context on the device named by LPM_B200_DEVICE (default 0).
lpm_ctx* context();

/// Throw the reference's exception type for a library status (no-op for LPM_OK).
void check(int status, const char* where);

/// lpm_kernel_desc of a reference vector kernel; throws std::logic_error("invalid kernel") for kernels
/// the GPU path does not implement.
lpm_kernel_desc describe(const VectorKernel& k);
/// lpm_kernel_desc of a scalar kernel (the reference's ScalarKernel subclasses and PoissonGreensFn3d).
lpm_kernel_desc describe(const ScalarKernel& k);

}  // namespace b200
}  // namespace Lpm

#endif
