// qoa_jit.h — run-time compiled complex128 tile passes (host side).
//
// A pass's op stream is known on the host before it runs. Instead of
// interpreting it (k_pass: op fetch, dispatch, run-time exchange addresses),
// the engine can emit the pass as straight-line CUDA C++ — every register
// bit, condition mask, exchange address and coefficient slot a literal — and
// compile it with NVRTC for sm_100a. Coefficient values stay kernel
// parameters (the PassParams travels as before), so the generated text, and
// the compiled kernel, depend only on the pass's structure: repeated circuits
// and circuits that differ only in angles reuse one kernel.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "qoa_kernels.cuh"

namespace qoa {

struct JitEntry;

// A compiled (or compiling) pass kernel.
class JitKernel {
public:
    JitKernel() = default;
    explicit JitKernel(std::shared_ptr<JitEntry> e) : e_(std::move(e)) {}
    bool ready() const;
    bool failed() const;
    // Launches the pass over the state: the same arguments as k_pass, plus
    // the handle's status words (a streamed pass sets bit 0 of status[0]
    // when a tile copy did not arrive in time). Grid 2^(n - TILE_BITS), or
    // for the streamed form one persistent CTA per resident slot.
    // amps: double2* (complex128 kernels) or float2* (complex64 kernels).
    cudaError_t launch(void* amps, const PassParams& P, const double* norm2_in, double* partials,
                       uint32_t* status, cudaStream_t st) const;
    // Arena form: njobs device ArenaJob records from `jobs`, 2^lt tiles each.
    cudaError_t launch_arena(const ArenaJob* jobs, uint32_t njobs, uint32_t lt, cudaStream_t st) const;

private:
    std::shared_ptr<JitEntry> e_;
};

// The kernel body (everything after the kernel's name) for a pass:
// complex128 (the k_pass form) or complex64 (the packed FP32 form of
// k_pass_p32).
// arena: the batch form, one launch over many jobs of this structure
// (ArenaJob list; CTA b runs tile b % 2^(n-11) of job b / 2^(n-11)).
std::string jit_pass_body(const PassParams& P, bool arena = false);
std::string jit_pass32_body(const PassParams& P, bool arena = false);

// Looks each body up in the process-wide cache; a missing one is compiled
// on the compile threads:
//   SECOND_SIGHTING  the second time it is requested (the first request
//                    returns an empty, never-ready kernel)
//   NOW              now, without waiting
//   WAIT             now, and the call returns when they are loaded
enum class JitWhen { SECOND_SIGHTING, NOW, WAIT };
std::vector<JitKernel> jit_request(const std::vector<std::string>& bodies, JitWhen when);

// The whole NVRTC program text for these bodies (prelude, kernels).
std::string jit_program(const std::vector<std::string>& bodies);

// Compiles the bodies with NVRTC without loading them (no GPU needed).
bool jit_compile_only(const std::vector<std::string>& bodies, std::string& err);

// Blocks until every submitted compile has finished.
void jit_wait_all();

struct JitStats {
    uint64_t kernels;      // compiled kernels in the cache
    uint64_t hits;         // requests served from the cache
    uint64_t misses;       // requests that started a compile
    uint64_t failures;     // kernels whose compile or load failed
    double compile_ms;     // total NVRTC + load time
};
JitStats jit_stats();

// Last compile error text (empty if none).
std::string jit_last_error();

}  // namespace qoa
