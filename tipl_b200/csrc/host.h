// Host-side runtime shared by the drivers and the C ABI: error reporting, device
// buffers on the stream-ordered allocator, the transform algebra.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>
#include "../../include/regb200.h"
#include "kernels.h"

namespace regb {

// Carries a regb_status out of deep host code; caught at the ABI boundary.
struct Failure : std::runtime_error {
    regb_status code;
    Failure(regb_status c, const std::string& what) : std::runtime_error(what), code(c) {}
};

void set_last_error(const std::string& s);
[[noreturn]] void throw_cuda(cudaError_t e, const char* what);

#define REGB_CK(x)                                  \
    do {                                            \
        cudaError_t e_ = (x);                       \
        if (e_ != cudaSuccess)                      \
            ::regb::throw_cuda(e_, #x);             \
    } while (0)

void ensure_device();  // pool release threshold etc., once per device

// Page-locked host blocks from a process-wide cache: cudaMallocHost / cudaFreeHost
// are slow and the free synchronises the device, so jobs that come and go reuse
// blocks instead.  pinned_get rounds `bytes` up to its size class (written back);
// pinned_put returns a block of that size.  pinned_trim frees every cached block.
void* pinned_get(size_t& bytes);
void pinned_put(void* p, size_t bytes);
void pinned_trim();

// Allocation-failure injection (regb_debug_fail_allocations): true when this device
// allocation of `bytes` bytes is one of those the hook was asked to fail.
bool alloc_fault_injected(size_t bytes);

// A device buffer from the stream-ordered pool (cudaMallocAsync); freed on the
// same stream, so reuse is ordered without device-wide synchronisation.
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t st = nullptr;
    DevBuf() = default;
    DevBuf(size_t count, cudaStream_t s) { alloc(count, s); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), st(o.st) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        if (this != &o) {
            reset();
            p = o.p;
            n = o.n;
            st = o.st;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    void alloc(size_t count, cudaStream_t s)
    {
        reset();
        ensure_device();
        st = s;
        n = count;
        if (count) {
            if (alloc_fault_injected(count * sizeof(T))) {
                n = 0;
                throw Failure(REGB_ERR_NOMEM, "device allocation failed: injected by regb_debug_fail_allocations");
            }
            cudaError_t e = cudaMallocAsync((void**)&p, count * sizeof(T), s);
            if (e != cudaSuccess) {
                p = nullptr;
                n = 0;
                (void)cudaGetLastError();
                throw Failure(REGB_ERR_NOMEM, std::string("device allocation failed: ") + cudaGetErrorString(e));
            }
        }
    }
    void zero() { REGB_CK(cudaMemsetAsync(p, 0, n * sizeof(T), st)); }
    void reset()
    {
        if (p)
            cudaFreeAsync(p, st);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { reset(); }
};

// Pinned host staging buffer.
template <typename T>
struct PinBuf {
    T* p = nullptr;
    size_t n = 0;
    PinBuf() = default;
    explicit PinBuf(size_t c) { alloc(c); }
    PinBuf(const PinBuf&) = delete;
    PinBuf& operator=(const PinBuf&) = delete;
    void alloc(size_t c)
    {
        if (c <= n)
            return;
        reset();
        bytes_ = c * sizeof(T);
        p = (T*)pinned_get(bytes_);  // bytes_ becomes the block's size class
        n = c;                       // the capacity callers see stays what they asked for
    }
    void reset()
    {
        if (p)
            pinned_put(p, bytes_);
        p = nullptr;
        n = 0;
        bytes_ = 0;
    }

private:
    size_t bytes_ = 0;

public:
    ~PinBuf() { reset(); }
};

// Owns a non-blocking stream.
struct Stream {
    cudaStream_t s = nullptr;
    Stream() { REGB_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~Stream()
    {
        if (s)
            cudaStreamDestroy(s);
    }
    Stream(const Stream&) = delete;
    Stream& operator=(const Stream&) = delete;
    void sync() { REGB_CK(cudaStreamSynchronize(s)); }
};

size_t pix_size(int dtype);

// ---- transform algebra (numerical/transformation.hpp) ----
void affine_to_matrix(const float* param, const int* from_dim, const float* from_vs, const int* to_dim,
                      const float* to_vs, float* T);
void affine_to_matrix_f64(const double* param, const int* from_dim, const double* from_vs, const int* to_dim,
                          const double* to_vs, double* T);
bool matrix_inverse(float* T);
bool integer_shift(const float* T, int* shift);

// ---- whole-registration drivers ----
struct LinearResult {
    float cost = 0.0f;
    long long evals = 0;
};
// The affine search of tipl::reg::linear on device-resident uint8 volumes.
class AffineBatcher;
class CdmScheduler;
LinearResult linear_register(const uint8_t* d_from, const int* fdim, const float* from_vs, const uint8_t* d_to,
                             const int* tdim, const float* to_vs, float* arg, const regb_linear_param& p,
                             volatile const int* terminated, cudaStream_t st, AffineBatcher* batcher = nullptr);
// The same over npairs image pairs d_from[i] / d_to[i] (tipl::reg::linear with
// make_list(It), make_list(I): every from-volume of dims fdim, every to-volume of dims
// tdim); a candidate's cost is the sum over pairs divided by 2 * npairs.
LinearResult linear_register_multi(const uint8_t* const* d_from, const uint8_t* const* d_to, int npairs,
                                   const int* fdim, const float* from_vs, const int* tdim, const float* to_vs,
                                   float* arg, const regb_linear_param& p, volatile const int* terminated,
                                   cudaStream_t st, AffineBatcher* batcher = nullptr);

LinearResult linear_register_state(const uint8_t* d_from, const int* fdim, const float* from_vs, const uint8_t* d_to,
                                   const int* tdim, const float* to_vs, float* arg, const regb_runner_state& s,
                                   volatile const int* terminated, cudaStream_t st);
LinearResult linear_register_state_multi(const uint8_t* const* d_from, const uint8_t* const* d_to, int npairs,
                                         const int* fdim, const float* from_vs, const int* tdim, const float* to_vs,
                                         float* arg, const regb_runner_state& s, volatile const int* terminated,
                                         cudaStream_t st);
void runner_state_from_param(const int* fdim, const float* from_vs, const int* tdim, const float* to_vs,
                             const float* arg, const regb_linear_param& p, regb_runner_state& s);

// The CDM driver (reg/cdm.hpp:373-474) on device-resident images of nmod modality
// pairs d_It[i] / d_Is[i] (one shape and pixel type); modality i uses gradient type
// gtypes[i] ('r' / 'd'; 'r' past the string's end).  d_field receives the
// full-resolution field (xyz per voxel).  ndim 2: the images are 2-D (dim[2] == 1)
// and the reference's dimension-2 instantiation is followed (the pyramid stops on
// min(w, h); the field's z stays 0).  Returns REGB_OK, REGB_FALSE or REGB_CANCELLED.
regb_status cdm_register_multi(const void* const* d_It, const void* const* d_Is, int nmod, const char* gtypes,
                               const int* dim, int pix, float* d_field, const regb_cdm_param& p,
                               volatile const int* terminated, cudaStream_t st, int* iterations = nullptr,
                               CdmScheduler* sched = nullptr, int ndim = 3);
// accumulate_displacement(dis, new_dis) (numerical/dif.hpp:166-186) on device fields of
// one shape: new_dis <- dis composed with new_dis.
void accumulate_displacement_device(const float* dis, float* new_dis, const int* dim, cudaStream_t st);
// One modality pair with p.gradient_type.
regb_status cdm_register(const void* d_It, const void* d_Is, const int* dim, int pix, float* d_field,
                         const regb_cdm_param& p, volatile const int* terminated, cudaStream_t st,
                         int* iterations = nullptr, CdmScheduler* sched = nullptr);

}  // namespace regb
