// gprat::GP and gprat::GP_data — same names, constructors and methods as the
// reference (core/include/gprat_c.hpp:21-228), computed by libgprat_cuda.so
// (include/gprat_cu.h) on a B200.  Inputs are copied at construction, as in
// the reference; every method call refactorises K with the current kernel
// parameters (the reference keeps nothing between calls either).
//
// Additions (no counterpart in the reference): predict_full_covariance,
// loss_and_gradient and set_precision.
#ifndef GPRAT_B200_GPRAT_C_HPP
#define GPRAT_B200_GPRAT_C_HPP

#include "gp_hyperparameters.hpp"
#include "gp_kernels.hpp"
#include "target.hpp"

#include <array>
#include <memory>
#include <string>
#include <vector>

struct gprat_cu_gp;

namespace gprat
{

struct GP_data
{
    std::string file_path;
    int n_samples;
    int n_regressors;
    std::vector<double> data;

    /** Loads n samples, prefixed with n_reg - 1 zeros (core/src/gprat_c.cpp:15-21). */
    GP_data(const std::string &file_path, int n, int n_reg);
};

class GP
{
  private:
    std::vector<double> training_input_;
    std::vector<double> training_output_;
    int n_tiles_;
    int n_tile_size_;
    std::vector<bool> trainable_params_;
    std::shared_ptr<Target> target_;
    std::shared_ptr<gprat_cu_gp> device_;
    int precision_ = 0;

    gprat_cu_gp *handle();
    std::array<double, 3> hyper() const;

  public:
    int n_reg;
    gprat_hyper::SEKParams kernel_params;

    GP(std::vector<double> input,
       std::vector<double> output,
       int n_tiles,
       int n_tile_size,
       int n_regressors,
       std::vector<double> kernel_hyperparams,
       std::vector<bool> trainable_bool,
       std::shared_ptr<Target> target);

    GP(std::vector<double> input,
       std::vector<double> output,
       int n_tiles,
       int n_tile_size,
       int n_regressors,
       std::vector<double> kernel_hyperparams,
       std::vector<bool> trainable_bool);

    GP(std::vector<double> input,
       std::vector<double> output,
       int n_tiles,
       int n_tile_size,
       int n_regressors,
       std::vector<double> kernel_hyperparams,
       std::vector<bool> trainable_bool,
       int gpu_id,
       int n_streams);

    std::string repr() const;

    std::vector<double> get_training_input() const;

    std::vector<double> get_training_output() const;

    std::vector<double> predict(const std::vector<double> &test_data, int m_tiles, int m_tile_size);

    std::vector<std::vector<double>>
    predict_with_uncertainty(const std::vector<double> &test_data, int m_tiles, int m_tile_size);

    /** Mean and the diagonal of the posterior covariance (as the reference returns). */
    std::vector<std::vector<double>>
    predict_with_full_cov(const std::vector<double> &test_data, int m_tiles, int m_tile_size);

    std::vector<double> optimize(const gprat_hyper::AdamParams &adam_params);

    double optimize_step(gprat_hyper::AdamParams &adam_params, int iter);

    double calculate_loss();

    /** n_tiles^2 row-major tiles; upper tiles are empty, diagonal tiles keep
     * K's strict upper triangle (as the reference returns). */
    std::vector<std::vector<double>> cholesky();

    /** {mean (m), posterior covariance (m*m, row-major)} for the first m
     * test points.  Addition: the reference discards all but the diagonal. */
    std::vector<std::vector<double>> predict_full_covariance(const std::vector<double> &test_data, int m);

    /** {loss, dloss/du_l, dloss/du_v, dloss/du_noise} at the current kernel
     * parameters (u = softplus^-1 of each parameter, reference scaling). */
    std::vector<double> loss_and_gradient();

    /** 0 = FP64 (default); see GPRAT_CU_PREC_* in gprat_cu.h. */
    void set_precision(int precision);
};

}  // namespace gprat

#endif
