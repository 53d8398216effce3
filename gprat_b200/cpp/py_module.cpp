// Python module `gprat` — the reference's Python API (bindings/gprat_py.cpp:10-142,
// bindings/utils_py.cpp:16-109, bindings/module.cpp:9-20) over gprat::GP.
//
// Same classes, constructor overloads (CPU constructor first), argument
// names, defaults and methods.  Additions: SEKParams is a bound type (the
// reference exposes kernel_params without binding its type), GP.cholesky,
// GP.predict_full_covariance, GP.loss_and_gradient and GP.set_precision.
#include "gprat_c.hpp"
#include "target.hpp"
#include "utils_c.hpp"

#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

namespace py = pybind11;

namespace
{

void start_hpx_wrapper(std::vector<std::string> args, std::size_t n_cores)
{
    if (args.empty())
    {
        args.push_back("gprat");
    }
    args.push_back("--hpx:threads=" + std::to_string(n_cores));
    std::vector<char *> argv;
    for (auto &a : args)
    {
        argv.push_back(a.data());
    }
    argv.push_back(nullptr);
    utils::start_hpx_runtime(static_cast<int>(args.size()), argv.data());
}

}  // namespace

PYBIND11_MODULE(gprat, m)
{
    m.doc() = "GPRat library (B200 / sm_100a implementation)";

    py::class_<gprat::GP_data>(m, "GP_data", "Class representing Gaussian Process data.")
        .def(py::init<std::string, int, int>(), py::arg("file_path"), py::arg("n_samples"), py::arg("n_regressors"),
             "Loads n_samples values from file_path, prefixed with n_regressors - 1 zeros.")
        .def_readonly("n_samples", &gprat::GP_data::n_samples)
        .def_readonly("n_regressors", &gprat::GP_data::n_regressors)
        .def_readonly("file_path", &gprat::GP_data::file_path)
        .def_readonly("data", &gprat::GP_data::data);

    py::class_<gprat_hyper::AdamParams>(m, "AdamParams")
        .def(py::init<double, double, double, double, int>(), py::arg("learning_rate") = 0.001,
             py::arg("beta1") = 0.9, py::arg("beta2") = 0.999, py::arg("epsilon") = 1e-8, py::arg("opt_iter") = 0)
        .def_readwrite("learning_rate", &gprat_hyper::AdamParams::learning_rate)
        .def_readwrite("beta1", &gprat_hyper::AdamParams::beta1)
        .def_readwrite("beta2", &gprat_hyper::AdamParams::beta2)
        .def_readwrite("epsilon", &gprat_hyper::AdamParams::epsilon)
        .def_readwrite("opt_iter", &gprat_hyper::AdamParams::opt_iter)
        .def("__repr__", &gprat_hyper::AdamParams::repr);

    py::class_<gprat_hyper::SEKParams>(m, "SEKParams")
        .def(py::init<double, double, double>(), py::arg("lengthscale"), py::arg("vertical_lengthscale"),
             py::arg("noise_variance"))
        .def_readwrite("lengthscale", &gprat_hyper::SEKParams::lengthscale)
        .def_readwrite("vertical_lengthscale", &gprat_hyper::SEKParams::vertical_lengthscale)
        .def_readwrite("noise_variance", &gprat_hyper::SEKParams::noise_variance)
        .def_readwrite("m_T", &gprat_hyper::SEKParams::m_T)
        .def_readwrite("w_T", &gprat_hyper::SEKParams::w_T)
        .def("__repr__",
             [](const gprat_hyper::SEKParams &p)
             {
                 return "SEKParams(lengthscale=" + std::to_string(p.lengthscale) +
                        ", vertical_lengthscale=" + std::to_string(p.vertical_lengthscale) +
                        ", noise_variance=" + std::to_string(p.noise_variance) + ")";
             });

    py::class_<gprat::GP>(m, "GP")
        .def(py::init<std::vector<double>, std::vector<double>, int, int, int, std::vector<double>,
                      std::vector<bool>>(),
             py::arg("input_data"), py::arg("output_data"), py::arg("n_tiles"), py::arg("n_tile_size"),
             py::arg("n_reg") = 8, py::arg("kernel_params") = std::vector<double>{ 1.0, 1.0, 0.1 },
             py::arg("trainable") = std::vector<bool>{ true, true, true },
             "Gaussian process on the current CUDA device.")
        .def(py::init<std::vector<double>, std::vector<double>, int, int, int, std::vector<double>, std::vector<bool>,
                      int, int>(),
             py::arg("input_data"), py::arg("output_data"), py::arg("n_tiles"), py::arg("n_tile_size"),
             py::arg("n_reg") = 8, py::arg("kernel_params") = std::vector<double>{ 1.0, 1.0, 0.1 },
             py::arg("trainable") = std::vector<bool>{ true, true, true }, py::arg("gpu_id") = 0,
             py::arg("n_streams") = 1, "Gaussian process on CUDA device gpu_id.")
        .def_readwrite("n_reg", &gprat::GP::n_reg)
        .def_readwrite("kernel_params", &gprat::GP::kernel_params)
        .def("__repr__", &gprat::GP::repr)
        .def("get_input_data", &gprat::GP::get_training_input)
        .def("get_output_data", &gprat::GP::get_training_output)
        .def("predict", &gprat::GP::predict, py::arg("test_data"), py::arg("m_tiles"), py::arg("m_tile_size"))
        .def("predict_with_uncertainty", &gprat::GP::predict_with_uncertainty, py::arg("test_data"),
             py::arg("m_tiles"), py::arg("m_tile_size"))
        .def("predict_with_full_cov", &gprat::GP::predict_with_full_cov, py::arg("test_data"), py::arg("m_tiles"),
             py::arg("m_tile_size"))
        .def("optimize", &gprat::GP::optimize, py::arg("AdamParams"))
        .def("optimize_step", &gprat::GP::optimize_step, py::arg("AdamParams"), py::arg("iter"))
        .def("compute_loss", &gprat::GP::calculate_loss)
        .def("cholesky", &gprat::GP::cholesky)
        .def("predict_full_covariance", &gprat::GP::predict_full_covariance, py::arg("test_data"), py::arg("m"))
        .def("loss_and_gradient", &gprat::GP::loss_and_gradient)
        .def("set_precision", &gprat::GP::set_precision, py::arg("precision"));

    m.def("compute_train_tiles", &utils::compute_train_tiles, py::arg("n_samples"), py::arg("n_tile_size"));
    m.def("compute_train_tile_size", &utils::compute_train_tile_size, py::arg("n_samples"), py::arg("n_tiles"));
    m.def("compute_test_tiles", &utils::compute_test_tiles, py::arg("m_samples"), py::arg("n_tiles"),
          py::arg("n_tile_size"));
    m.def("print_vector", &utils::print_vector, py::arg("vec"), py::arg("start") = 0, py::arg("end") = -1,
          py::arg("separator") = " ");
    m.def("start_hpx", &start_hpx_wrapper, py::arg("args"), py::arg("n_cores"));
    m.def("resume_hpx", &utils::resume_hpx_runtime);
    m.def("suspend_hpx", &utils::suspend_hpx_runtime);
    m.def("stop_hpx", &utils::stop_hpx_runtime);
    m.def("compiled_with_cuda", &utils::compiled_with_cuda);
    m.def("print_available_gpus", &gprat::print_available_gpus);
    m.def("gpu_count", &gprat::gpu_count);
}
