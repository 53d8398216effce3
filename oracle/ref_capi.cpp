// Test infrastructure (oracle build only).  A C entry layer over the
// reference's own gprat::GP class (core/include/gprat_c.hpp:54-228), compiled
// together with the reference's unmodified CPU sources into
// oracle/_ref/libgprat_ref.so.  Tests and the CPU baseline call it through
// ctypes (oracle/ref.py).  Every function returns 0 on success and -1 after
// an exception, whose text is available from gprat_ref_last_error().
#include "gprat_c.hpp"
#include "utils_c.hpp"

#include <cstring>
#include <string>
#include <vector>

extern "C" void scipy_openblas_set_num_threads(int);

namespace
{
thread_local std::string g_last_error;

struct RefGP
{
    gprat::GP gp;
};

template <typename F>
int guarded(F &&f)
{
    try
    {
        f();
        return 0;
    }
    catch (const std::exception &e)
    {
        g_last_error = e.what();
    }
    catch (...)
    {
        g_last_error = "unknown exception";
    }
    return -1;
}
}  // namespace

extern "C" {

const char *gprat_ref_last_error() { return g_last_error.c_str(); }

// Starts the task runtime with n_threads workers (HPX: --hpx:threads=N).
int gprat_ref_start(int n_threads)
{
    return guarded(
        [&]
        {
            scipy_openblas_set_num_threads(1);
            std::string a0 = "gprat";
            std::string a1 = "--hpx:threads=" + std::to_string(n_threads);
            char *argv[] = { a0.data(), a1.data(), nullptr };
            utils::start_hpx_runtime(2, argv);
        });
}

int gprat_ref_stop() { return guarded([] { utils::stop_hpx_runtime(); }); }

void *gprat_ref_create(const double *x,
                       long nx,
                       const double *y,
                       long ny,
                       int n_tiles,
                       int n_tile_size,
                       int n_reg,
                       double lengthscale,
                       double vertical_lengthscale,
                       double noise_variance,
                       int train_l,
                       int train_v,
                       int train_n)
{
    RefGP *out = nullptr;
    guarded(
        [&]
        {
            std::vector<double> in(x, x + nx);
            std::vector<double> outv(y, y + ny);
            out = new RefGP{ gprat::GP(in,
                                       outv,
                                       n_tiles,
                                       n_tile_size,
                                       n_reg,
                                       { lengthscale, vertical_lengthscale, noise_variance },
                                       { train_l != 0, train_v != 0, train_n != 0 }) };
        });
    return out;
}

void gprat_ref_destroy(void *h) { delete static_cast<RefGP *>(h); }

// params: lengthscale, vertical_lengthscale, noise_variance, m_T[3], w_T[3]
int gprat_ref_get_params(void *h, double *params)
{
    return guarded(
        [&]
        {
            auto &kp = static_cast<RefGP *>(h)->gp.kernel_params;
            params[0] = kp.lengthscale;
            params[1] = kp.vertical_lengthscale;
            params[2] = kp.noise_variance;
            for (int i = 0; i < 3; ++i)
            {
                params[3 + i] = kp.m_T[static_cast<std::size_t>(i)];
                params[6 + i] = kp.w_T[static_cast<std::size_t>(i)];
            }
        });
}

int gprat_ref_set_params(void *h, const double *params)
{
    return guarded(
        [&]
        {
            auto &kp = static_cast<RefGP *>(h)->gp.kernel_params;
            kp.lengthscale = params[0];
            kp.vertical_lengthscale = params[1];
            kp.noise_variance = params[2];
            for (int i = 0; i < 3; ++i)
            {
                kp.m_T[static_cast<std::size_t>(i)] = params[3 + i];
                kp.w_T[static_cast<std::size_t>(i)] = params[6 + i];
            }
        });
}

// out: n_tiles^2 tiles of n_tile_size^2 doubles, tile (i,j) at offset
// (i*n_tiles+j)*T*T; tiles the reference leaves empty (upper) are zero-filled
// and flagged 0 in `present` (n_tiles^2 bytes).
int gprat_ref_cholesky(void *h, double *out, unsigned char *present)
{
    return guarded(
        [&]
        {
            auto tiles = static_cast<RefGP *>(h)->gp.cholesky();
            std::size_t off = 0;
            std::size_t tile_elems = 0;
            for (auto &t : tiles)
            {
                tile_elems = std::max(tile_elems, t.size());
            }
            for (std::size_t k = 0; k < tiles.size(); ++k)
            {
                present[k] = tiles[k].empty() ? 0 : 1;
                if (tiles[k].empty())
                {
                    std::memset(out + off, 0, tile_elems * sizeof(double));
                }
                else
                {
                    std::memcpy(out + off, tiles[k].data(), tiles[k].size() * sizeof(double));
                }
                off += tile_elems;
            }
        });
}

int gprat_ref_predict(void *h, const double *xt, long nxt, int m_tiles, int m_tile_size, double *mean)
{
    return guarded(
        [&]
        {
            std::vector<double> test(xt, xt + nxt);
            auto r = static_cast<RefGP *>(h)->gp.predict(test, m_tiles, m_tile_size);
            std::memcpy(mean, r.data(), r.size() * sizeof(double));
        });
}

int gprat_ref_predict_with_uncertainty(
    void *h, const double *xt, long nxt, int m_tiles, int m_tile_size, double *mean, double *var)
{
    return guarded(
        [&]
        {
            std::vector<double> test(xt, xt + nxt);
            auto r = static_cast<RefGP *>(h)->gp.predict_with_uncertainty(test, m_tiles, m_tile_size);
            std::memcpy(mean, r[0].data(), r[0].size() * sizeof(double));
            std::memcpy(var, r[1].data(), r[1].size() * sizeof(double));
        });
}

int gprat_ref_predict_with_full_cov(
    void *h, const double *xt, long nxt, int m_tiles, int m_tile_size, double *mean, double *var)
{
    return guarded(
        [&]
        {
            std::vector<double> test(xt, xt + nxt);
            auto r = static_cast<RefGP *>(h)->gp.predict_with_full_cov(test, m_tiles, m_tile_size);
            std::memcpy(mean, r[0].data(), r[0].size() * sizeof(double));
            std::memcpy(var, r[1].data(), r[1].size() * sizeof(double));
        });
}

int gprat_ref_calculate_loss(void *h, double *loss)
{
    return guarded([&] { *loss = static_cast<RefGP *>(h)->gp.calculate_loss(); });
}

int gprat_ref_optimize(void *h, double lr, double b1, double b2, double eps, int opt_iter, double *losses)
{
    return guarded(
        [&]
        {
            gprat_hyper::AdamParams adam(lr, b1, b2, eps, opt_iter);
            auto r = static_cast<RefGP *>(h)->gp.optimize(adam);
            std::memcpy(losses, r.data(), r.size() * sizeof(double));
        });
}

int gprat_ref_optimize_step(void *h, double lr, double b1, double b2, double eps, int opt_iter, int iter, double *loss)
{
    return guarded(
        [&]
        {
            gprat_hyper::AdamParams adam(lr, b1, b2, eps, opt_iter);
            *loss = static_cast<RefGP *>(h)->gp.optimize_step(adam, iter);
        });
}

int gprat_ref_compute_test_tiles(int n_test, int n_tiles, int n_tile_size, int *m_tiles, int *m_tile_size)
{
    return guarded(
        [&]
        {
            auto p = utils::compute_test_tiles(n_test, n_tiles, n_tile_size);
            *m_tiles = p.first;
            *m_tile_size = p.second;
        });
}

}  // extern "C"
