// mw_serial.cu -- a flat byte image of a device tree: checkpoint files and messages between processes.
//
// Contract: FunctionTree::saveTree / loadTree as used for orbital checkpoints at reference
// src/qmfunctions/Orbital.cpp:118-190, and the payload of mrcpp::send_tree / recv_tree
// (src/parallel.cpp:208-232).  The image (all fields little-endian, 8-byte aligned):
//   bytes  0-7   magic "MWB2TREE"
//          8-11  uint32 format version (1)
//         12-15  int32 k (scaling functions per dimension)
//         16-19  int32 basis type (0 interpolating, 1 Legendre)
//         20-23  int32 root scale n0
//         24-35  int32 corner[3]
//         36-47  int32 boxes[3]
//         48-55  int64 n (nodes)
//         56-63  reserved (0)
//   then int64 trans[3n], float64 coef[n (2k)^3], int32 depth[n], parent[n], child0[n], in the node
//   layout of include/mwb200.h (parents before children).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mwb200.h"
#include "mw_internal.hpp"

namespace mwb {
void set_last_error(const std::string& msg);
}

struct mw_tree_s : mwb::Tree {};

namespace {

constexpr char kMagic[8] = {'M', 'W', 'B', '2', 'T', 'R', 'E', 'E'};
constexpr uint32_t kVersion = 1;
constexpr size_t kHeader = 64;

struct Header {
    char magic[8];
    uint32_t version;
    int32_t k, basis, n0, corner[3], boxes[3];
    int64_t n;
    int64_t reserved;
};
static_assert(sizeof(Header) == kHeader, "header layout");

size_t image_bytes(const mwb::Tree& t) {
    const size_t n = (size_t)t.n;
    return kHeader + n * (3 * 8 + t.mra->bsize() * 8 + 3 * 4);
}

void check_world(const Header& h, const mwb::Mra& m) {
    if (std::memcmp(h.magic, kMagic, 8) != 0) throw mwb::Error(MW_ERR_ARG, "not a tree image (bad magic)");
    if (h.version != kVersion) throw mwb::Error(MW_ERR_ARG, "unsupported tree image version");
    bool same = h.k == m.k && h.basis == m.basis.type && h.n0 == m.n0;
    for (int d = 0; d < 3; ++d) same = same && h.corner[d] == m.corner[d] && h.boxes[d] == m.boxes[d];
    if (!same) throw mwb::Error(MW_ERR_ARG, "tree image was written on a different world or basis");
    if (h.n <= 0 || h.n > (1LL << 31) - 1) throw mwb::Error(MW_ERR_ARG, "bad node count in tree image");
}

void write_image(mw_tree t, unsigned char* buf) {
    const mwb::Mra& m = *t->mra;
    Header h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.k = m.k;
    h.basis = m.basis.type;
    h.n0 = m.n0;
    for (int d = 0; d < 3; ++d) {
        h.corner[d] = m.corner[d];
        h.boxes[d] = m.boxes[d];
    }
    h.n = t->n;
    std::memcpy(buf, &h, kHeader);
    const size_t n = (size_t)t->n, BS = m.bsize();
    auto* trans = reinterpret_cast<long long*>(buf + kHeader);
    auto* coef = reinterpret_cast<double*>(buf + kHeader + 3 * 8 * n);
    auto* ints = reinterpret_cast<int*>(buf + kHeader + 3 * 8 * n + 8 * BS * n);
    const int st = mw_tree_download(t, ints, trans, ints + n, ints + 2 * n, coef);
    if (st != MW_OK) throw mwb::Error(st, mw_last_error());
}

void read_image(mw_tree t, const unsigned char* buf, size_t len) {
    if (len < kHeader) throw mwb::Error(MW_ERR_ARG, "tree image too short");
    Header h;
    std::memcpy(&h, buf, kHeader);
    check_world(h, *t->mra);
    const size_t n = (size_t)h.n, BS = t->mra->bsize();
    if (len < kHeader + n * (3 * 8 + BS * 8 + 3 * 4)) throw mwb::Error(MW_ERR_ARG, "tree image truncated");
    const auto* trans = reinterpret_cast<const long long*>(buf + kHeader);
    const auto* coef = reinterpret_cast<const double*>(buf + kHeader + 3 * 8 * n);
    const auto* ints = reinterpret_cast<const int*>(buf + kHeader + 3 * 8 * n + 8 * BS * n);
    const int st = mw_tree_upload(t, (int)n, ints, trans, ints + n, ints + 2 * n, coef);
    if (st != MW_OK) throw mwb::Error(st, mw_last_error());
}

}  // namespace

#define MWS_TRY(...)                                \
    try {                                           \
        __VA_ARGS__;                                \
        return MW_OK;                               \
    } catch (const mwb::Error& e) {                 \
        mwb::set_last_error(e.what());              \
        return e.code;                              \
    } catch (const std::exception& e) {             \
        mwb::set_last_error(e.what());              \
        return MW_ERR_STATE;                        \
    }

extern "C" {

int mw_tree_serialized_size(mw_tree t, unsigned long long* bytes) {
    MWS_TRY({
        if (!t || !bytes) throw mwb::Error(MW_ERR_ARG, "null pointer");
        if (t->n == 0) throw mwb::Error(MW_ERR_STATE, "empty tree");
        *bytes = image_bytes(*t);
    })
}

int mw_tree_serialize(mw_tree t, void* buf, unsigned long long cap) {
    MWS_TRY({
        if (!t || !buf) throw mwb::Error(MW_ERR_ARG, "null pointer");
        if (t->n == 0) throw mwb::Error(MW_ERR_STATE, "empty tree");
        if (cap < image_bytes(*t)) throw mwb::Error(MW_ERR_CAPACITY, "buffer smaller than mw_tree_serialized_size");
        write_image(t, static_cast<unsigned char*>(buf));
    })
}

int mw_tree_deserialize(mw_tree t, const void* buf, unsigned long long len) {
    MWS_TRY({
        if (!t || !buf) throw mwb::Error(MW_ERR_ARG, "null pointer");
        read_image(t, static_cast<const unsigned char*>(buf), (size_t)len);
    })
}

int mw_tree_save(mw_tree t, const char* path) {
    MWS_TRY({
        if (!t || !path) throw mwb::Error(MW_ERR_ARG, "null pointer");
        if (t->n == 0) throw mwb::Error(MW_ERR_STATE, "empty tree");
        std::vector<unsigned char> img(image_bytes(*t));
        write_image(t, img.data());
        FILE* f = std::fopen(path, "wb");
        if (!f) throw mwb::Error(MW_ERR_ARG, std::string("cannot open for writing: ") + path);
        const size_t w = std::fwrite(img.data(), 1, img.size(), f);
        const int c = std::fclose(f);
        if (w != img.size() || c != 0) throw mwb::Error(MW_ERR_STATE, std::string("write failed: ") + path);
    })
}

int mw_tree_load(mw_tree t, const char* path) {
    MWS_TRY({
        if (!t || !path) throw mwb::Error(MW_ERR_ARG, "null pointer");
        FILE* f = std::fopen(path, "rb");
        if (!f) throw mwb::Error(MW_ERR_ARG, std::string("cannot open for reading: ") + path);
        std::vector<unsigned char> img;
        unsigned char chunk[1 << 16];
        size_t r;
        while ((r = std::fread(chunk, 1, sizeof(chunk), f)) > 0) img.insert(img.end(), chunk, chunk + r);
        std::fclose(f);
        read_image(t, img.data(), img.size());
    })
}

}  // extern "C"
