// Shared pieces of the drop-in classes: the library context, status -> exception mapping and kernel
// descriptors read from the reference's kernel objects.
#include "LpmB200Dropin.h"

#include <cstdlib>
#include <mutex>
#include <new>
#include <stdexcept>

namespace Lpm {
namespace b200 {

lpm_ctx* context() {
    static std::once_flag once;
    static lpm_ctx* ctx = nullptr;
    static int status = LPM_OK;
    std::call_once(once, [] {
        const char* s = std::getenv("LPM_B200_DEVICE");
        status = lpm_ctx_create(s ? std::atoi(s) : 0, &ctx);
    });
    check(status, "lpm_ctx_create");
    return ctx;
}

void check(int status, const char* where) {
    if (status == LPM_OK) return;
    const std::string msg = std::string(where) + ": " + lpm_last_error();
    if (status == LPM_ERR_OOM) throw std::bad_alloc();
    if (status == LPM_ERR_KERNEL) throw std::logic_error("invalid kernel");
    throw std::runtime_error(msg);
}

lpm_kernel_desc describe(const VectorKernel& k) {
    lpm_kernel_desc d{};
    if (!dynamic_cast<const BiotSavartSphere*>(&k)) throw std::logic_error("invalid kernel");
    // BiotSavartSphere keeps delta and R protected: recover them from its public interface.
    // sumMultiplier() = -1/(4 pi R); at x = (R,0,0), y = (0,R,0): K_z = R^2 / (R^2 + delta^2).
    const double R = -1.0 / (4.0 * PI * k.sumMultiplier());
    const XyzVector kz = k.evaluate(XyzVector(R, 0.0, 0.0), XyzVector(0.0, R, 0.0));
    const double d2 = R * R / kz.z - R * R;
    d.kind = LPM_KERNEL_BIOT_SAVART_SPHERE;
    d.radius = R;
    d.delta = k.isSingular() ? 0.0 : std::sqrt(d2 > 0.0 ? d2 : 0.0);
    return d;
}

lpm_kernel_desc describe(const ScalarKernel& k) {
    lpm_kernel_desc d{};
    if (!dynamic_cast<const PoissonGreensFn3d*>(&k)) throw std::logic_error("invalid kernel");
    d.kind = LPM_KERNEL_POISSON_3D;
    d.radius = 1.0;
    d.delta = 0.0;
    return d;
}

}  // namespace b200
}  // namespace Lpm
