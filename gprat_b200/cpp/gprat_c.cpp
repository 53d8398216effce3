// gprat::GP and gprat::GP_data over the C ABI of libgprat_cuda.so.
//
// Mirrors the reference's core/src/gprat_c.cpp:15-361: same constructors,
// same method names, arguments, return shapes and exception types.  Every
// method runs on the GP's CUDA device through include/gprat_cu.h; there is
// no CPU path (a GP built with the CPU target runs on the current CUDA
// device).  Failures map to C++ exceptions: invalid arguments to
// std::invalid_argument, everything else (no device, CUDA errors, a
// covariance matrix that is not positive definite) to std::runtime_error.
#include "gprat_c.hpp"

#include "gprat_cu.h"
#include "utils_c.hpp"

#include <iomanip>
#include <sstream>
#include <stdexcept>

namespace gprat
{
namespace
{

void check(int rc)
{
    if (rc == GPRAT_CU_OK)
    {
        return;
    }
    std::string msg = gprat_cu_last_error();
    if (rc == GPRAT_CU_ERR_INVALID_ARG)
    {
        throw std::invalid_argument(msg);
    }
    throw std::runtime_error(msg);
}

std::vector<int> trainable_ints(const std::vector<bool> &t)
{
    std::vector<int> out(3, 0);
    for (std::size_t i = 0; i < 3 && i < t.size(); ++i)
    {
        out[i] = t[i] ? 1 : 0;
    }
    return out;
}

}  // namespace

GP_data::GP_data(const std::string &f_path, int n, int n_reg) : file_path(f_path), n_samples(n), n_regressors(n_reg)
{
    data = utils::load_data(f_path, n, n_reg - 1);
}

static gprat_hyper::SEKParams make_params(const std::vector<double> &h)
{
    if (h.size() < 3)
    {
        throw std::invalid_argument("kernel_params must hold lengthscale, vertical_lengthscale, noise_variance");
    }
    return gprat_hyper::SEKParams(h[0], h[1], h[2]);
}

GP::GP(std::vector<double> input,
       std::vector<double> output,
       int n_tiles,
       int n_tile_size,
       int n_regressors,
       std::vector<double> kernel_hyperparams,
       std::vector<bool> trainable_bool,
       std::shared_ptr<Target> target) :
    training_input_(std::move(input)),
    training_output_(std::move(output)),
    n_tiles_(n_tiles),
    n_tile_size_(n_tile_size),
    trainable_params_(std::move(trainable_bool)),
    target_(std::move(target)),
    n_reg(n_regressors),
    kernel_params(make_params(kernel_hyperparams))
{ }

GP::GP(std::vector<double> input,
       std::vector<double> output,
       int n_tiles,
       int n_tile_size,
       int n_regressors,
       std::vector<double> kernel_hyperparams,
       std::vector<bool> trainable_bool) :
    GP(std::move(input),
       std::move(output),
       n_tiles,
       n_tile_size,
       n_regressors,
       std::move(kernel_hyperparams),
       std::move(trainable_bool),
       std::make_shared<CPU>())
{ }

GP::GP(std::vector<double> input,
       std::vector<double> output,
       int n_tiles,
       int n_tile_size,
       int n_regressors,
       std::vector<double> kernel_hyperparams,
       std::vector<bool> trainable_bool,
       int gpu_id,
       int n_streams) :
    GP(std::move(input),
       std::move(output),
       n_tiles,
       n_tile_size,
       n_regressors,
       std::move(kernel_hyperparams),
       std::move(trainable_bool),
       std::make_shared<CUDA_GPU>(gpu_id, n_streams))
{ }

gprat_cu_gp *GP::handle()
{
    if (!device_)
    {
        gprat_cu_gp *h = nullptr;
        check(gprat_cu_gp_create(target_->device(),
                                 training_input_.data(),
                                 static_cast<int64_t>(training_input_.size()),
                                 training_output_.data(),
                                 static_cast<int64_t>(training_output_.size()),
                                 n_tiles_,
                                 n_tile_size_,
                                 n_reg,
                                 &h));
        device_ = std::shared_ptr<gprat_cu_gp>(h, [](gprat_cu_gp *p) { gprat_cu_gp_destroy(p); });
        if (precision_ != GPRAT_CU_PREC_FP64)
        {
            check(gprat_cu_gp_set_precision(h, precision_));
        }
    }
    return device_.get();
}

std::array<double, 3> GP::hyper() const
{
    return { kernel_params.lengthscale, kernel_params.vertical_lengthscale, kernel_params.noise_variance };
}

std::string GP::repr() const
{
    std::ostringstream oss;
    oss << std::fixed << std::setprecision(12);
    oss << "Kernel_Params: [lengthscale=" << kernel_params.lengthscale
        << ", vertical_lengthscale=" << kernel_params.vertical_lengthscale
        << ", noise_variance=" << kernel_params.noise_variance << ", n_regressors=" << n_reg
        << "], Trainable_Params: [trainable_params l=" << trainable_params_[0]
        << ", trainable_params v=" << trainable_params_[1] << ", trainable_params n=" << trainable_params_[2]
        << "], Target: [" << target_->repr() << "], n_tiles=" << n_tiles_ << ", n_tile_size=" << n_tile_size_;
    return oss.str();
}

std::vector<double> GP::get_training_input() const { return training_input_; }

std::vector<double> GP::get_training_output() const { return training_output_; }

std::vector<double> GP::predict(const std::vector<double> &test_data, int m_tiles, int m_tile_size)
{
    const auto h = hyper();
    std::vector<double> mean(static_cast<std::size_t>(std::max(0, m_tiles * m_tile_size)));
    check(gprat_cu_predict(handle(), h.data(), test_data.data(), static_cast<int64_t>(test_data.size()), m_tiles,
                           m_tile_size, mean.data()));
    return mean;
}

std::vector<std::vector<double>>
GP::predict_with_uncertainty(const std::vector<double> &test_data, int m_tiles, int m_tile_size)
{
    const auto h = hyper();
    const std::size_t m = static_cast<std::size_t>(std::max(0, m_tiles * m_tile_size));
    std::vector<double> mean(m), var(m);
    check(gprat_cu_predict_with_uncertainty(handle(), h.data(), test_data.data(),
                                            static_cast<int64_t>(test_data.size()), m_tiles, m_tile_size, mean.data(),
                                            var.data()));
    return { std::move(mean), std::move(var) };
}

std::vector<std::vector<double>>
GP::predict_with_full_cov(const std::vector<double> &test_data, int m_tiles, int m_tile_size)
{
    const auto h = hyper();
    const std::size_t m = static_cast<std::size_t>(std::max(0, m_tiles * m_tile_size));
    std::vector<double> mean(m), var(m);
    check(gprat_cu_predict_with_full_cov(handle(), h.data(), test_data.data(), static_cast<int64_t>(test_data.size()),
                                         m_tiles, m_tile_size, mean.data(), var.data()));
    return { std::move(mean), std::move(var) };
}

std::vector<double> GP::optimize(const gprat_hyper::AdamParams &adam_params)
{
    double params[9] = { kernel_params.lengthscale, kernel_params.vertical_lengthscale, kernel_params.noise_variance,
                         kernel_params.m_T[0],      kernel_params.m_T[1],                kernel_params.m_T[2],
                         kernel_params.w_T[0],      kernel_params.w_T[1],                kernel_params.w_T[2] };
    const double adam[4] = { adam_params.learning_rate, adam_params.beta1, adam_params.beta2, adam_params.epsilon };
    const auto trainable = trainable_ints(trainable_params_);
    std::vector<double> losses(static_cast<std::size_t>(std::max(0, adam_params.opt_iter)));
    check(gprat_cu_optimize(handle(), params, adam, trainable.data(), adam_params.opt_iter, losses.data()));
    kernel_params.lengthscale = params[0];
    kernel_params.vertical_lengthscale = params[1];
    kernel_params.noise_variance = params[2];
    for (int q = 0; q < 3; ++q)
    {
        kernel_params.m_T[static_cast<std::size_t>(q)] = params[3 + q];
        kernel_params.w_T[static_cast<std::size_t>(q)] = params[6 + q];
    }
    return losses;
}

double GP::optimize_step(gprat_hyper::AdamParams &adam_params, int iter)
{
    double params[9] = { kernel_params.lengthscale, kernel_params.vertical_lengthscale, kernel_params.noise_variance,
                         kernel_params.m_T[0],      kernel_params.m_T[1],                kernel_params.m_T[2],
                         kernel_params.w_T[0],      kernel_params.w_T[1],                kernel_params.w_T[2] };
    const double adam[4] = { adam_params.learning_rate, adam_params.beta1, adam_params.beta2, adam_params.epsilon };
    const auto trainable = trainable_ints(trainable_params_);
    double loss = 0.0;
    check(gprat_cu_optimize_step(handle(), params, adam, trainable.data(), iter, &loss));
    kernel_params.lengthscale = params[0];
    kernel_params.vertical_lengthscale = params[1];
    kernel_params.noise_variance = params[2];
    for (int q = 0; q < 3; ++q)
    {
        kernel_params.m_T[static_cast<std::size_t>(q)] = params[3 + q];
        kernel_params.w_T[static_cast<std::size_t>(q)] = params[6 + q];
    }
    return loss;
}

double GP::calculate_loss()
{
    const auto h = hyper();
    double loss = 0.0;
    check(gprat_cu_compute_loss(handle(), h.data(), &loss));
    return loss;
}

std::vector<std::vector<double>> GP::cholesky()
{
    const auto h = hyper();
    const std::size_t nt = static_cast<std::size_t>(n_tiles_);
    const std::size_t tt = static_cast<std::size_t>(n_tile_size_) * static_cast<std::size_t>(n_tile_size_);
    std::vector<double> all(nt * nt * tt);
    check(gprat_cu_cholesky(handle(), h.data(), all.data()));
    std::vector<std::vector<double>> tiles(nt * nt);
    for (std::size_t i = 0; i < nt; ++i)
    {
        for (std::size_t j = 0; j <= i; ++j)
        {
            const double *src = all.data() + (i * nt + j) * tt;
            tiles[i * nt + j].assign(src, src + tt);
        }
    }
    return tiles;
}

std::vector<std::vector<double>> GP::predict_full_covariance(const std::vector<double> &test_data, int m)
{
    const auto h = hyper();
    const std::size_t mm = static_cast<std::size_t>(std::max(0, m));
    std::vector<double> mean(mm), cov(mm * mm);
    check(gprat_cu_predict_full_covariance(handle(), h.data(), test_data.data(),
                                           static_cast<int64_t>(test_data.size()), m, mean.data(), cov.data()));
    return { std::move(mean), std::move(cov) };
}

std::vector<double> GP::loss_and_gradient()
{
    const auto h = hyper();
    double loss = 0.0;
    double grad[3] = { 0.0, 0.0, 0.0 };
    check(gprat_cu_loss_grad(handle(), h.data(), &loss, grad));
    return { loss, grad[0], grad[1], grad[2] };
}

void GP::set_precision(int precision)
{
    if (device_)
    {
        check(gprat_cu_gp_set_precision(device_.get(), precision));
    }
    else if (precision != GPRAT_CU_PREC_FP64 && precision != GPRAT_CU_PREC_MIXED_TF32 &&
             precision != GPRAT_CU_PREC_MIXED_BF16)
    {
        throw std::invalid_argument("unknown precision mode");
    }
    precision_ = precision;
}

}  // namespace gprat
