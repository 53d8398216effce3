// Adam optimiser settings (same type and members as the reference's
// gprat_hyper::AdamParams, core/include/gp_hyperparameters.hpp:12-56).
#ifndef GPRAT_B200_GP_HYPERPARAMETERS_HPP
#define GPRAT_B200_GP_HYPERPARAMETERS_HPP

#include <string>

namespace gprat_hyper
{

struct AdamParams
{
    double learning_rate;
    double beta1;
    double beta2;
    double epsilon;
    /** Number of iterations run by GP::optimize. */
    int opt_iter;

    AdamParams(double lr = 0.001, double b1 = 0.9, double b2 = 0.999, double eps = 1e-8, int opt_i = 0);

    std::string repr() const;
};

}  // namespace gprat_hyper

#endif
