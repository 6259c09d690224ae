// checkpoint.cuh -- CPD-ALS checkpoint files.
//
// A checkpoint holds the ALS loop state after a whole iteration: the factor
// matrices as the loop keeps them (each column divided by the weight of the
// solve that produced it), the weights of the last mode's solve, and the fit
// after every iteration so far.  Resuming from it repeats what the
// uninterrupted loop would have done next: the iteration count selects the
// column-max weights rule and the BF16/FP32 schedule, and the last fit is the
// one the tolerance test compares against.
//
// File layout (little-endian, every section a multiple of 8 bytes):
//   header (48 bytes)  char magic[8] = "PTICPDCK"; u32 version = 1, nmodes,
//                      rank, iters, flags (bit 0: the loop had converged),
//                      reserved; u64 nnz; f64 sum of squared values
//   u32 ndims[nmodes]  zero-padded to an even count
//   f64 fits[iters]
//   f32 lambda[rank], then each mode's factor, ndims[m] x rank row-major;
//                      zero-padded to a multiple of 8 bytes
//   u64 checksum       FNV-1a over the preceding file as 64-bit words
//                      (h = 0xcbf29ce484222325; h ^= w; h *= 0x100000001b3)
// A file is written as <path>.tmp and renamed over <path>, so a crash while
// writing leaves the previous checkpoint in place.
#pragma once
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace pti {

constexpr char kCkptMagic[8] = {'P', 'T', 'I', 'C', 'P', 'D', 'C', 'K'};
constexpr uint32_t kCkptVersion = 1;
constexpr uint32_t kCkptConverged = 1;

struct CkptState {
    uint32_t nmodes = 0, rank = 0, iters = 0, flags = 0;
    uint64_t nnz = 0;
    double normX2 = 0.0;
    std::vector<uint32_t> ndims;
    std::vector<double> fits;
    std::vector<float> lambda;
    std::vector<std::vector<float>> factors;  // ndims[m] x rank each
};

// Reads and verifies a checkpoint.  A missing file sets *missing (when given)
// and returns 0 with `st` untouched; any other failure is an error.
int ckpt_read(const char *path, CkptState &st, bool *missing);

// Writes checkpoints of one ALS run.  save() enqueues the device-to-host
// copies of the state on the ALS stream and returns; a background thread
// waits for them and writes the file, so the loop keeps running.  The next
// save() (and finish()) first waits for the previous write.
class CkptWriter {
public:
    CkptWriter() = default;
    CkptWriter(const CkptWriter &) = delete;
    CkptWriter &operator=(const CkptWriter &) = delete;
    ~CkptWriter();

    int init(const char *path, uint32_t nmodes, const uint32_t *ndims, uint64_t nnz, uint32_t rank,
             uint32_t max_iters);
    // State after `iters` iterations: factors A[m] (stride floats per row),
    // lambda (rank floats), fits (device, iters doubles), normX2 (device).
    int save(float *const *A, uint32_t stride, const float *lambda, const double *fits, const double *normX2,
             uint32_t iters, bool converged, cudaStream_t s);
    // Waits for the last write and reports its failure, if any.
    int finish();

private:
    void write_file();

    std::string path_;
    std::vector<uint32_t> ndims_;
    uint64_t nnz_ = 0;
    uint32_t rank_ = 0, max_iters_ = 0, iters_ = 0, flags_ = 0;
    size_t factor_floats_ = 0;
    unsigned char *host_ = nullptr;  // pinned: normX2, fits[max_iters], lambda, factors
    cudaEvent_t ev_ = nullptr;
    std::thread th_;
    int err_ = 0;
    std::string why_;
};

}  // namespace pti
