// gprat_hyper::SEKParams and gprat_hyper::AdamParams (interface of the
// reference's core/src/gp_kernels.cpp:7-53 and core/src/gp_hyperparameters.cpp:9-31).
#include "gp_hyperparameters.hpp"
#include "gp_kernels.hpp"

#include <iomanip>
#include <sstream>
#include <stdexcept>

namespace gprat_hyper
{

SEKParams::SEKParams(double lengthscale_, double vertical_lengthscale_, double noise_variance_) :
    lengthscale(lengthscale_),
    vertical_lengthscale(vertical_lengthscale_),
    noise_variance(noise_variance_),
    m_T(3, 0.0),
    w_T(3, 0.0)
{ }

std::size_t SEKParams::size() { return 3; }

void SEKParams::set_param(std::size_t index, double value)
{
    switch (index)
    {
        case 0: lengthscale = value; return;
        case 1: vertical_lengthscale = value; return;
        case 2: noise_variance = value; return;
        default: throw std::invalid_argument("Set Invalid param_idx");
    }
}

const double &SEKParams::get_param(std::size_t index) const
{
    switch (index)
    {
        case 0: return lengthscale;
        case 1: return vertical_lengthscale;
        case 2: return noise_variance;
        default: throw std::invalid_argument("Get Invalid param_idx");
    }
}

AdamParams::AdamParams(double lr, double b1, double b2, double eps, int opt_i) :
    learning_rate(lr),
    beta1(b1),
    beta2(b2),
    epsilon(eps),
    opt_iter(opt_i)
{ }

std::string AdamParams::repr() const
{
    std::ostringstream oss;
    oss << std::fixed << std::setprecision(8) << "Hyperparameters: [learning_rate=" << learning_rate
        << ", beta1=" << beta1 << ", beta2=" << beta2 << ", epsilon=" << epsilon << ", opt_iter=" << opt_iter << "]";
    return oss.str();
}

}  // namespace gprat_hyper
