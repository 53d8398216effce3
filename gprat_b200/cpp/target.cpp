// Compute targets (interface of the reference's core/src/target.cpp:13-157).
#include "target.hpp"

#include "gprat_cu.h"

#include <cuda_runtime.h>

#include <iostream>
#include <sstream>
#include <stdexcept>

namespace gprat
{

CPU::CPU() { }

bool CPU::is_cpu() { return true; }

bool CPU::is_gpu() { return false; }

std::string CPU::repr() const { return "CPU"; }

int CPU::device() const
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
    {
        cudaGetLastError();
        dev = 0;
    }
    return dev;
}

CPU get_cpu() { return CPU(); }

CUDA_GPU::CUDA_GPU(int id_, int n_streams_) : id(id_), n_streams(n_streams_), i_stream(0), shared_memory_size(0)
{
    if (id < 0 || id >= gpu_count())
    {
        throw std::runtime_error("Requested GPU device is not available.");
    }
}

bool CUDA_GPU::is_cpu() { return false; }

bool CUDA_GPU::is_gpu() { return true; }

std::string CUDA_GPU::repr() const
{
    std::ostringstream oss;
    oss << "GPU (CUDA): [id=" << id << ", n_streams=" << n_streams << "]";
    return oss.str();
}

int CUDA_GPU::device() const { return id; }

CUDA_GPU get_gpu(int id, int n_streams) { return CUDA_GPU(id, n_streams); }

CUDA_GPU get_gpu() { return CUDA_GPU(0, 1); }

void print_available_gpus()
{
    const int count = gpu_count();
    for (int i = 0; i < count; ++i)
    {
        cudaDeviceProp p{};
        if (cudaGetDeviceProperties(&p, i) != cudaSuccess)
        {
            continue;
        }
        std::cout << "Device " << i << ": " << p.name << "\n"
                  << "  Total Global Memory: " << p.totalGlobalMem << "\n"
                  << "  Shared Memory per Block: " << p.sharedMemPerBlock << "\n"
                  << "  Max Threads per Block: " << p.maxThreadsPerBlock << "\n"
                  << "  Total Constant Memory: " << p.totalConstMem << "\n"
                  << "  Compute Capability: " << p.major << "." << p.minor << "\n"
                  << "  Multiprocessor Count: " << p.multiProcessorCount << "\n"
                  << "  Memory Bus Width: " << p.memoryBusWidth << " bits" << std::endl;
    }
}

int gpu_count()
{
    int count = 0;
    if (gprat_cu_device_count(&count) != GPRAT_CU_OK)
    {
        return 0;
    }
    return count;
}

}  // namespace gprat
