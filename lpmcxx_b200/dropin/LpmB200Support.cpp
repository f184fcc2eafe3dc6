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
    d.radius = 1.0;
    d.delta = 0.0;
    const XyzVector ex(1.0, 0.0, 0.0), zero(0.0, 0.0, 0.0);
    if (dynamic_cast<const PoissonGreensFn3d*>(&k)) {
        d.kind = LPM_KERNEL_POISSON_3D;
    } else if (dynamic_cast<const SphereGreensFn*>(&k)) {
        // the radius is protected: K(x,y) = -log(R^2 - x.y)/(4 pi R), so K at x.y = -1 minus K at x.y = 0
        // is -log(1 + 1/R^2)/(4 pi R), strictly increasing in R > 0: bisection in log R brackets R; Newton
        // steps on K(0, 0) = -log(R)/(2 pi R) then restore full precision where that equation is well
        // conditioned (away from R = e, the extremum of log(R)/R)
        const double k00 = k.evaluate(zero, zero);
        const double g = k.evaluate(ex, -1.0 * ex) - k00;
        double lo = std::log(1e-8), hi = std::log(1e8);
        for (int it = 0; it < 200 && hi - lo > 1e-15; ++it) {
            const double mid = 0.5 * (lo + hi), R = std::exp(mid);
            if (-std::log1p(1.0 / (R * R)) / (4.0 * PI * R) < g) lo = mid;
            else hi = mid;
        }
        double R = std::exp(0.5 * (lo + hi));
        if (std::fabs(std::log(R) - 1.0) > 0.5) {
            for (int it = 0; it < 4; ++it) {
                const double h = -std::log(R) / (2.0 * PI * R) - k00;
                const double dh = -(1.0 - std::log(R)) / (2.0 * PI * R * R);
                R -= h / dh;
            }
        }
        d.kind = LPM_KERNEL_SPHERE_GREENS;
        d.radius = R;
    } else if (dynamic_cast<const PlanarGreensFnFreeBoundaries*>(&k)) {
        d.kind = LPM_KERNEL_PLANAR_LOG;
    } else if (dynamic_cast<const SecondOrderDelta3d*>(&k)) {
        // K(x, x) = 3/(4 pi eps^3)
        d.kind = LPM_KERNEL_DELTA_3D;
        d.delta = std::cbrt(3.0 / (4.0 * PI * k.evaluate(ex, ex)));
    } else if (dynamic_cast<const SphereDelta*>(&k)) {
        // K(x, x) on the unit sphere = 1/(2 pi eps^2) - 1/(4 pi)
        d.kind = LPM_KERNEL_SPHERE_DELTA;
        d.delta = std::sqrt(1.0 / (2.0 * PI * (k.evaluate(ex, ex) + 1.0 / (4.0 * PI))));
    } else {
        throw std::logic_error("invalid kernel");
    }
    return d;
}

}  // namespace b200
}  // namespace Lpm
