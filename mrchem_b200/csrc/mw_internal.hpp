// mw_internal.hpp -- host-side objects behind the C-ABI handles (include/mwb200.h).
#pragma once
#include <initializer_list>
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "mw_math.hpp"

namespace mwb {

// error carried to the C-ABI boundary (converted to a status code + mw_last_error text)
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define MWB_CUDA(call)                                                                           \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            throw ::mwb::Error(-2, std::string(#call) + ": " + cudaGetErrorString(e_) + " (" +    \
                                       __FILE__ + ":" + std::to_string(__LINE__) + ")");          \
    } while (0)

constexpr int kKeyBits = 19;          // translation bits per dimension in a node key
constexpr uint64_t kEmptyKey = ~0ull; // empty hash slot

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int num_sms = 0;
    // profiling counters (benchmarks): kernels of this library launched, and CUDA-event time of
    // the contraction kernel when enabled
    bool prof = false;
    long long launches = 0;
    long long apply_launches = 0;
    long long apply_ctas = 0;  // CTAs (chunks) of those launches
    double apply_ms = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // contraction work per CTA: at most this many (output, input, term) triples, per engine (FP64, FP32,
    // split-TF32, BF16x3 tensor-core x step); set by the caller or an autotuner (load balance against partial-block traffic)
    int chunk_triples[4] = {48, 48, 48, 48};
    // handles that point here (worlds, networks); a destroyed context is freed with the last of them
    int refs = 0;
    bool closed = false;
    // small host<->device transfers of the passes go through mapped pinned host memory and are moved by
    // copy kernels, not by the DMA copy engines: the engines may be busy with large tree transfers of
    // other contexts (a caller streaming batches), and a small copy queued behind them would wait.
    // Uploads: a staging arena, a region reused only after the event recorded behind the latest copy
    // kernel that read it completed.  Read-backs: a mailbox written by a copy kernel before the sync.
    char* pin = nullptr;      // host address
    char* pin_dev = nullptr;  // its device address
    size_t pin_cap = 0, pin_off = 0;
    cudaEvent_t pin_ev = nullptr;
    bool pin_pending = false;
    char* mbox = nullptr;
    char* mbox_dev = nullptr;
    size_t mbox_cap = 0;
};

struct Mra {
    Ctx* ctx = nullptr;
    int n0 = 0;
    int corner[3] = {0, 0, 0};
    int boxes[3] = {1, 1, 1};
    int max_depth = 0;      // as requested (sets the operators' r_min)
    int depth_limit = 0;    // max_depth clamped to the key capacity
    int k = 0;
    ScalingBasis basis;
    std::vector<double> F;  // (2k)^2 two-scale filter
    std::vector<double> W;  // k x k projection quadrature matrix
    double* d_F = nullptr;   // F
    double* d_FT = nullptr;  // F^T
    double* d_PF = nullptr;  // projection matrix F * blkdiag(W, W)
    double* d_MV = nullptr;  // evaluation matrix blkdiag(E, E) * F^T (pointwise product)
    // trees and operators that point here; a destroyed world is freed with the last of them
    int refs = 0;
    bool closed = false;
    size_t bsize() const { return (size_t)8 * k * k * k; }
};

// Per-depth operator tables (device layout documented in mw_kernels.cuh)
struct DeltaRec {
    int d[3];
    int t0, t1;
    int lrank;  // dz rank << 10 | dy rank among the depth's offsets (line order of the contraction)
    double maxb;
};
struct TermRec {
    int mx, my, mz, m;
    double beta;
    double bound;
};

struct OpDepth {
    std::vector<double> mats;          // NS matrices, (2k)^2 each
    std::vector<DeltaRec> deltas;      // sorted by maxb, descending
    std::vector<TermRec> terms;
    double* d_mats = nullptr;
    float* d_mats32 = nullptr;  // FP32 copy of d_mats (mixed-precision apply)
    double* d_matsb = nullptr;  // each matrix scaled by its term's beta (z-step operators)
    float* d_matsb32 = nullptr;
    // the same four tables transposed and zero-padded to P x P (P = 2k rounded up to a multiple of
    // 4), entry [k][o] = M[o][k]: the layout the GEMM-tiled contraction copies into shared memory
    double* d_matsT = nullptr;
    float* d_matsT32 = nullptr;
    double* d_matsbT = nullptr;
    float* d_matsbT32 = nullptr;
    // split-TF32 operator images for the tensor-core contraction: per matrix one K-major FP32 image of
    // 3 KP8 rows and KP8 columns (KP8 = 2k rounded up to a multiple of 8, zero padding): rows o,
    // KP8 + o, 2 KP8 + o = hi, mid, lo TF32 pieces of M[o][.]; entry (row n, k) at word
    // 4 (n + 3 KP8 (k / 4)) + k % 4; plain and beta-scaled
    float* d_matsI = nullptr;
    float* d_matsbI = nullptr;
    // tensor-core x step with CUDA-core y and z steps (k_happly, 2k <= 20 only): the FP32 transposed
    // operators in the split column layout of its y/z tiles (entry [k][split_pos(o, P/4, 4)] = M[o][k]),
    // plain and beta-scaled, and per matrix one image of its three BF16 slices (mw_slice.hpp, XGeo::OPB
    // bytes)
    float* d_matsS32 = nullptr;
    float* d_matsbS32 = nullptr;
    unsigned char* d_matsX = nullptr;
    DeltaRec* d_deltas = nullptr;
    TermRec* d_terms = nullptr;
};

struct Op {
    Mra* mra = nullptr;
    int kind = 0;                  // 0: separated-Gaussian convolution; 1: first derivative (ABGV)
    double da = 0.0, db = 0.0;     // derivative flux parameters
    std::vector<double> dT[3];     // derivative unit-scale blocks T(-1), T(0), T(1), k x k
    double mu = 0.0, prec = 0.0, eps = 0.0;
    std::vector<GaussTerm> terms;
    std::unique_ptr<GaussianOperatorBuilder> builder;
    double B0 = 0.0;
    std::map<int, std::unique_ptr<OpDepth>> depths;
    std::mutex mtx;
    ~Op();
};

struct Tree {
    Mra* mra = nullptr;
    int n = 0, cap = 0;
    uint64_t* key = nullptr;
    int* parent = nullptr;
    int* child0 = nullptr;
    double* coef = nullptr;
    double* norm2 = nullptr;   // squared norm of the whole block
    double* wnorm2 = nullptr;  // squared norm of the wavelet part
    uint64_t* hkey = nullptr;
    int* hval = nullptr;
    uint32_t hcap = 0;
    std::vector<int> level_begin;  // level d = [level_begin[d], level_begin[d+1])
    long long stats[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double g0 = 0.0;      // root-level norm of the last apply into this tree (sets its thresholds)
    double prec = 0.0;    // precision of the last apply into this tree
    ~Tree();
    int levels() const { return (int)level_begin.size() - 1; }
};

// device memory from the stream-ordered pool
void* dalloc(Ctx* ctx, size_t bytes);
void dfree(Ctx* ctx, void* p);
// stream-ordered copy of `bytes` host bytes to device memory `dst` through the context's pinned arena
// (pageable copy when the arena cannot hold them); the host buffer may be reused when this returns
void upload_bytes(Ctx* ctx, void* dst, const void* src, size_t bytes);
// the same on stream s: through the arena when s is the context's stream, else a pageable copy on s
void upload_bytes(Ctx* ctx, cudaStream_t s, void* dst, const void* src, size_t bytes);
// device-to-device copy on the context's stream by a copy kernel (the DMA engines may be queued with
// large host transfers of other contexts)
void device_copy(Ctx* ctx, void* dst, const void* src, size_t bytes);
// synchronous read-back of several device ranges into host memory: one copy kernel into the mapped
// mailbox, a stream synchronisation, then host copies (a range that does not fit the mailbox goes
// through the copy engine)
struct ReadReq {
    void* dst;        // host
    const void* src;  // device
    size_t bytes;
};
void readback(Ctx* ctx, std::initializer_list<ReadReq> reqs);
// the same on stream s: through the mailbox when s is the context's stream, else copy-engine copies on s
void readback(Ctx* ctx, cudaStream_t s, std::initializer_list<ReadReq> reqs);

}  // namespace mwb
