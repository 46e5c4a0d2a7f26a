// mw_kernels.cuh -- launchers of the sm_100a kernels (mw_kernels.cu), called by the host driver.
#pragma once
#include <cstdint>
#include <vector>

#include "mw_internal.hpp"

namespace mwb {

// analytic function for projection (device copy of the parameter block)
struct FuncDesc {
    int type;
    int nterm;
    const double* p;
};

// Transform modes of launch_transform_nodes
enum TransformMode {
    TM_PROJECT = 0,   // quadrature block of f at the node -> compressed block
    TM_COMPRESS = 1,  // children's scaling parts -> compressed block of the parent
    TM_SUMUP = 2,     // reconstruct parent block, add the child parts into the children's scaling parts
};

// Per-apply view of the input tree for the candidate and contraction kernels
struct InView {
    const uint64_t* hkey;
    const int* hval;
    uint32_t hcap;
    const double* coef;
    const double* norm2;
};

// d_nodes == nullptr: the node range [begin, begin + nnodes) (compress / sum-up skip leaves)
void launch_transform_nodes(Tree& t, int mode, const int* d_nodes, int nnodes, const FuncDesc* f, cudaStream_t s,
                            int begin = 0);
void launch_node_norms(Tree& t, int begin, int end, cudaStream_t s);
// sum-up top-down, compress bottom-up and/or node norms of several trees, one launch per level
void trees_finish(const std::vector<Tree*>& ts, bool sumup, bool compress, bool norms, cudaStream_t s);
void launch_hash_reset(Tree& t, cudaStream_t s);
void launch_hash_insert(Tree& t, int begin, int end, cudaStream_t s);
// flags[i - begin] = sqrt(wnorm2[i]) > thr(depth) for i in [begin, end); returns number of splits
// and writes the split list (tree indices) to d_list
int launch_split(Tree& t, int begin, int end, int depth, double thr, int depth_limit, int* d_list,
                 cudaStream_t s);
// append 8 children for each node in d_list (n_split entries)
void launch_make_children(Tree& t, const int* d_list, int nsplit, cudaStream_t s);
// append 8 children for every node in lists[i] of tree ts[i] (one level per tree), enter them into the
// hash indices and push the new level start; one launch for all trees
void trees_add_children(const std::vector<Tree*>& ts, const std::vector<std::vector<int>>& lists, cudaStream_t s);
// internal node list of [begin, end) (returns count)
int launch_internal_list(Tree& t, int begin, int end, int* d_list, cudaStream_t s);
// deterministic reductions: sum of norm2 over leaves (or over [begin,end) when all=true), max norm2
double reduce_leaf_norm2(Tree& t, cudaStream_t s);
double reduce_range_norm2(Tree& t, int begin, int end, cudaStream_t s);
double reduce_max_norm2(Tree& t, cudaStream_t s);
void reduce_norms_many(const std::vector<Tree*>& ts, std::vector<double>& leaf2, std::vector<double>& max2,
                       cudaStream_t s);
void launch_rescale(Tree& t, double c, cudaStream_t s);
double launch_dot(Tree& a, Tree& b, cudaStream_t s);
double launch_distance(Tree& a, Tree& b, cudaStream_t s);
// dst[i] = src[perm[i]] for n blocks of bs doubles
void launch_gather_blocks(const double* src, const int* perm, int n, size_t bs, double* dst, cudaStream_t s);

// tree bookkeeping shared by the drivers (mw_api.cu)
void tree_reserve(Tree& t, int need);
void tree_make_roots(Tree& t);
// the root level of several trees of one world at once (two launches for the batch)
void trees_make_roots(const std::vector<Tree*>& ts);
// rebuild the hash indices of several trees of one context from their node keys (two launches)
void trees_rehash(const std::vector<Tree*>& ts);
void tree_compress_bottom_up(Tree& t);
// split the nodes of the last level whose wavelet norm exceeds thr; returns the number of new nodes
int tree_refine_last_level(Tree& t, double thr);

// one refinement pass of a batched apply (mw_apply.cu)
struct BatchTree {
    Tree* out = nullptr;
    Tree* inp = nullptr;
    const OpDepth* tab = nullptr;
    int obegin = 0, oend = 0;  // output nodes of this depth
    int nprefix = 0;           // leading offset entries that can pass the screening
    double theta = 0.0;        // screening threshold
    double prec = 0.0;
    double g0 = 0.0;           // root-level output norm (set by the root pass)
    int depth = 0;             // depth of these output nodes
};
struct BatchPass {
    int precision = 0;  // 0: FP64 products, 1: FP32 products with FP64 accumulation
    std::vector<BatchTree> trees;
    long long triples = 0;
    int nitems = 0, nchunks = 0, nslots = 0;
    std::vector<std::vector<int>> split_lists;  // per entry: nodes to split (level order)
    // per item of the pass (entries in order, nodes in order): 1 if the node splits
    std::vector<int> split_flags;
};
void run_batch_pass(BatchPass& bp, cudaStream_t s);

}  // namespace mwb
