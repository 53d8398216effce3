// Squared-exponential kernel hyper-parameters (same type and members as the
// reference's gprat_hyper::SEKParams, core/include/gp_kernels.hpp:14-78).
#ifndef GPRAT_B200_GP_KERNELS_HPP
#define GPRAT_B200_GP_KERNELS_HPP

#include <cstddef>
#include <vector>

namespace gprat_hyper
{

struct SEKParams
{
    /** Lengthscale l of k(x,y) = v * exp(-|x-y|^2 / (2 l^2)) (index 0). */
    double lengthscale;
    /** Vertical lengthscale v: multiplies the kernel directly (index 1). */
    double vertical_lengthscale;
    /** Noise variance added on the diagonal of K (index 2). */
    double noise_variance;
    /** Adam first moments, one per parameter. */
    std::vector<double> m_T;
    /** Adam second moments, one per parameter. */
    std::vector<double> w_T;

    SEKParams(double lengthscale_, double vertical_lengthscale_, double noise_variance_);

    std::size_t size();

    /** Sets parameter 0, 1 or 2; std::invalid_argument otherwise. */
    void set_param(std::size_t index, double value);

    /** Returns parameter 0, 1 or 2; std::invalid_argument otherwise. */
    const double &get_param(std::size_t index) const;
};

}  // namespace gprat_hyper

#endif
