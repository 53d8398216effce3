// Compute targets (same names as the reference's core/include/target.hpp:22-204).
//
// Every computation of this library runs on a CUDA GPU; there is no CPU
// path.  A GP constructed with the CPU target runs on the current CUDA
// device (device 0 unless the caller selected another one).  CUDA_GPU keeps
// the reference's id / n_streams fields; each GP uses one CUDA stream of its
// own, so n_streams is recorded but does not change the computation, and the
// reference's per-stream cuBLAS handles do not exist here.
#ifndef GPRAT_B200_TARGET_HPP
#define GPRAT_B200_TARGET_HPP

#include <string>
#include <vector>

namespace gprat
{

struct Target
{
    virtual bool is_cpu() = 0;
    virtual bool is_gpu() = 0;
    virtual std::string repr() const = 0;
    virtual ~Target() { }

    /** CUDA device that executes GP calls made with this target. */
    virtual int device() const = 0;

  protected:
    Target() = default;
};

struct CPU : public Target
{
  public:
    CPU();
    bool is_cpu() override;
    bool is_gpu() override;
    std::string repr() const override;
    int device() const override;
};

CPU get_cpu();

struct CUDA_GPU : public Target
{
    int id;
    int n_streams;
    int i_stream;
    int shared_memory_size;

    /** Throws std::runtime_error("Requested GPU device is not available.")
     * when id is not a valid device (core/src/target.cpp:24-41). */
    CUDA_GPU(int id, int n_streams);

    bool is_cpu() override;
    bool is_gpu() override;
    std::string repr() const override;
    int device() const override;
};

CUDA_GPU get_gpu(int id, int n_streams);

CUDA_GPU get_gpu();

void print_available_gpus();

int gpu_count();

}  // namespace gprat

#endif
