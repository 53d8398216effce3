// Utility functions (semantics of the reference's core/src/utils_c.cpp:8-140).
#include "utils_c.hpp"

#include <cstdio>
#include <iostream>
#include <stdexcept>

namespace utils
{

int compute_train_tiles(int n_samples, int n_tile_size)
{
    if (n_tile_size > 0)
    {
        return n_samples / n_tile_size;
    }
    throw std::runtime_error("Error: Please specify a valid value for train_tile_size.\n");
}

int compute_train_tile_size(int n_samples, int n_tiles)
{
    if (n_tiles > 0)
    {
        return n_samples / n_tiles;
    }
    throw std::runtime_error("Error: Please specify a valid value for train_tiles.\n");
}

std::pair<int, int> compute_test_tiles(int n_test, int n_tiles, int n_tile_size)
{
    if (n_tile_size <= 0 || n_tiles <= 0)
    {
        throw std::runtime_error("Error: n_tiles and n_tile_size must be positive.\n");
    }
    if ((n_test % n_tile_size) > 0)
    {
        return { n_tiles, n_test / n_tiles };
    }
    return { n_test / n_tile_size, n_tile_size };
}

std::vector<double> load_data(const std::string &file_path, int n_samples, int offset)
{
    std::vector<double> data(static_cast<std::size_t>(n_samples + offset), 0.0);
    FILE *f = std::fopen(file_path.c_str(), "r");
    if (f == nullptr)
    {
        throw std::runtime_error("Error: File not found: " + file_path);
    }
    int scanned = 0;
    for (int i = 0; i < n_samples; ++i)
    {
        scanned += std::fscanf(f, "%lf", &data[static_cast<std::size_t>(i + offset)]);
    }
    std::fclose(f);
    if (scanned != n_samples)
    {
        throw std::runtime_error("Error: Data not correctly read. Expected " + std::to_string(n_samples) +
                                 " elements, but read " + std::to_string(scanned));
    }
    return data;
}

void print_vector(const std::vector<double> &vec, int start, int end, const std::string &separator)
{
    const int size = static_cast<int>(vec.size());
    if (start < 0)
    {
        start += size;
    }
    if (end < 0)
    {
        end += size + 1;
    }
    if (start < 0)
    {
        start = 0;
    }
    if (end > size)
    {
        end = size;
    }
    if (start >= size || start >= end)
    {
        std::cerr << "Invalid range" << std::endl;
        return;
    }
    for (int i = start; i < end; ++i)
    {
        std::cout << vec[static_cast<std::size_t>(i)];
        if (i < end - 1)
        {
            std::cout << separator;
        }
    }
    std::cout << std::endl;
}

void start_hpx_runtime(int, char **) { }

void resume_hpx_runtime() { }

void suspend_hpx_runtime() { }

void stop_hpx_runtime() { }

bool compiled_with_cuda() { return true; }

}  // namespace utils
