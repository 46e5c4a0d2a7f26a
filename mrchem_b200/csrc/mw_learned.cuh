// mw_learned.cuh -- learned tree proposal: MLP, features, training, tree rebuild (mw_learned.cu).
#pragma once
#include <vector>

#include "mw_internal.hpp"

namespace mwb {

constexpr int kNF = 64;  // features per candidate output node

struct Mlp {
    Ctx* ctx = nullptr;
    int nhidden = 3, width = 128;
    std::vector<int> dims;           // kNF, width x nhidden, 1
    std::vector<size_t> woff, boff;  // offsets of W_l (out x in, row-major) and b_l in the parameters
    size_t nparam = 0;
    float* d_p = nullptr;            // parameters
    float* d_m = nullptr;            // Adam moments
    float* d_v = nullptr;
    float* d_g = nullptr;            // gradient of the last backward
    long long adam_t = 0;
    float* d_X = nullptr;            // training set (device): features and labels
    float* d_y = nullptr;
    int n_data = 0, cap_data = 0;
    ~Mlp();
};

struct FeatCtx {
    Tree* out;
    Tree* inp;
    Op* op;
    double prec, g0;
};

void mlp_init(Mlp& M, Ctx* ctx, int nhidden, int width, unsigned seed);
void mlp_forward(Mlp& M, const float* d_X, int N, std::vector<float*>& acts, cudaStream_t s);
double mlp_backward(Mlp& M, std::vector<float*>& acts, const float* d_y, const float* d_w, int N, cudaStream_t s);
void free_acts(Mlp& M, std::vector<float*>& acts);
std::vector<float> mlp_logits(Mlp& M, const float* d_X, int N, cudaStream_t s);
double mlp_train(Mlp& M, int epochs, int batch, float lr, unsigned seed);
void mlp_append(Mlp& M, const float* d_F, const std::vector<float>& y, cudaStream_t s);
// device features (n x kNF) of output nodes items[i] = (feature context index, node)
float* features(Ctx* ctx, std::vector<FeatCtx>& fc, const std::vector<int2>& items, cudaStream_t s);
void trees_rebuild(const std::vector<Tree*>& ts, const std::vector<std::vector<char>>& keeps,
                   const std::vector<std::vector<uint64_t>>& keys);
// Exact criterion over every node of the trees, on the device: keep[off[i] + q] = 1 when every strict
// ancestor of node q of tree i splits (sqrt(wnorm2) > thr[i][depth], depth < depth_limit); a kept node
// that splits but has no children is a miss.  Returns the misses as (tree, node, key) triples in no
// particular order.  d_keep must hold sum(n) bytes.
struct Miss {
    int tree, node;
    uint64_t key;
};
std::vector<Miss> verify_trees(const std::vector<Tree*>& ts, const std::vector<std::vector<double>>& thr,
                               int depth_limit, unsigned char* d_keep, cudaStream_t s);
// Rebuild every tree from its kept nodes (d_keep as written by verify_trees for the same trees),
// ordered by key (parents before children, level-contiguous), on the device; one synchronisation.
// Returns the number of nodes dropped.
long long trees_rebuild_device(const std::vector<Tree*>& ts, const unsigned char* d_keep, cudaStream_t s);
uint64_t host_make_key(int depth, long long tx, long long ty, long long tz);
void host_key_trans(uint64_t k, long long t[3]);

}  // namespace mwb
