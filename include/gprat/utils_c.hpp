// Utility functions (same names and semantics as the reference's
// core/include/utils_c.hpp:19-86).  The HPX runtime controls are kept for
// source compatibility: this library has no task runtime to start, so they
// only record the requested thread count.
#ifndef GPRAT_B200_UTILS_C_HPP
#define GPRAT_B200_UTILS_C_HPP

#include <string>
#include <utility>
#include <vector>

namespace utils
{

/** n_samples / n_tile_size; std::runtime_error if n_tile_size <= 0. */
int compute_train_tiles(int n_samples, int n_tile_size);

/** n_samples / n_tiles; std::runtime_error if n_tiles <= 0. */
int compute_train_tile_size(int n_samples, int n_tiles);

/** {m_tiles, m_tile_size}: same tile size if n_test is divisible by
 * n_tile_size, otherwise n_tiles tiles of n_test / n_tiles (truncating). */
std::pair<int, int> compute_test_tiles(int n_test, int n_tiles, int n_tile_size);

/** offset zeros followed by n_samples values read with %lf. */
std::vector<double> load_data(const std::string &file_path, int n_samples, int offset);

void print_vector(const std::vector<double> &vec, int start, int end, const std::string &separator);

void start_hpx_runtime(int argc, char **argv);
void resume_hpx_runtime();
void suspend_hpx_runtime();
void stop_hpx_runtime();

/** Always true: this library computes on CUDA GPUs. */
bool compiled_with_cuda();

}  // namespace utils

#endif
