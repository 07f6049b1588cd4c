// host.h -- host-side pieces of the miner (plain C++, no CUDA).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace qcb {

struct HostGraph {
    int32_t n = 0;
    std::vector<int64_t> off;  // n+1
    std::vector<int32_t> adj;  // sorted rows
    std::vector<int64_t> off2; // n+1 (empty until built)
    std::vector<int32_t> adj2;
};

// Parse the serialized graph (Mike12041204/cuQC main.cu:96-121 reads the
// same seven whitespace-separated sections with operator>>).  Returns "" on
// success, else a message.
std::string read_serialized(const char* path, HostGraph& g);
std::string write_serialized(const HostGraph& g, const char* path);

// Binary CSR file, for graphs too large for the text format to load quickly:
// 8 bytes "QCSRBIN1", then little-endian int64 n, nnz (= 2|E|) and nnz2 (the
// two-hop entries; -1 when the file holds no two-hop lists), then int64
// off[n+1], int32 adj[nnz], zero padding to a multiple of 8 bytes, and, when
// nnz2 >= 0, int64 off2[n+1] and int32 adj2[nnz2].
constexpr char kBinaryMagic[8] = {'Q', 'C', 'S', 'R', 'B', 'I', 'N', '1'};
bool is_binary_graph(const char* path);
std::string read_binary(const char* path, HostGraph& g, bool& has_twohop);
std::string write_binary(const HostGraph& g, const char* path);
// Structural checks the kernels rely on: offsets monotone, ids in range,
// rows sorted and duplicate-free, no self loops, symmetric 1-hop rows.
std::string validate(const HostGraph& g, bool need_twohop);

// md[k] = ceil(gamma*(k-1)) (main.cu:526-533) and ubt[d] = floor(d/gamma)
// (main.cu:1905), both in double exactly as the reference computes them.
void gamma_tables(double gamma, int n, int min_size, std::vector<int32_t>& md,
                  std::vector<int32_t>& ubt);

// Level 0 (main.cu:846-998): degree / 2-hop-size filter, iterated degree
// peeling, cover vertex and its covered neighbours, Q order.  Fills the root
// task's vertex ids (covered, candidates, cover) and the covered count.
void build_root(const HostGraph& g, const int32_t* md, int min_size, std::vector<int32_t>& ids,
                int& cov);

// Maximal sets of an emitted family [k, ids..]*: each sorted ascending,
// duplicates merged, sets with a proper superset in the family dropped,
// result in lexicographic order of the id sequences (the reference's prefix
// tree produces this order, main.cu:4881-4937).
void maximal_sets(const int32_t* flat, int64_t nints, std::vector<int32_t>& out, int64_t& nsets);

// "<k> v1 .. vk \n" lines (main.cu:4641-4652)
std::string write_result(const int32_t* flat, int64_t nints, const char* path);

} // namespace qcb
