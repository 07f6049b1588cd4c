// convert.cpp -- the graph-format tools of the cuQC pipeline, as one program
// (qc_convert) over the library's C ABI:
//
//   qc_convert edges2adj <edge_file> <0|1> [adj_out]
//       edge list ("u v" per line) -> adjacency list, one line per vertex
//       0..max id, neighbours in file order; 1 also adds every edge reversed.
//       Follows edgeToAdj.py (Mike12041204/cuQC edgeToAdj.py:5-50); writes to
//       stdout without adj_out, as the script prints.
//   qc_convert rmempty <adj_in> <adj_out>
//       drops the vertices with empty lines and renumbers the others in line
//       order (rmEmptyVert.py:29-63).
//   qc_convert adj2ser <adj_in> <ser_out>
//       adjacency list -> serialized graph with its two-hop lists, the
//       two-hop lists built on the GPU (adjToSer.cpp:45-204).
//   qc_convert adj2bin <adj_in> <bin_out> [0|1]
//       adjacency list -> binary CSR file, with the two-hop lists (1, the
//       default, built on the GPU) or without them (0: the reader builds them).
//   qc_convert ser2bin <ser_in> <bin_out>
//   qc_convert bin2ser <bin_in> <ser_out>
//
// Differences from the scripts: a malformed line (not two integers, a
// negative id) is an error instead of a Python exception; an id naming a
// vertex with an empty line in rmempty is an error (the script raises
// KeyError); adj2ser rejects characters other than digits, ' ' and '\n' (the
// reference parser folds them into numbers) and ids outside the graph (the
// reference indexes past its arrays).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/qc.h"

namespace {

bool read_file(const char* path, std::string& s)
{
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    s.clear();
    char buf[1 << 16];
    size_t k;
    while ((k = fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, k);
    fclose(f);
    return true;
}

void put_num(std::string& s, int64_t v)
{
    char b[24];
    int n = 0;
    const bool neg = v < 0;
    uint64_t u = neg ? (uint64_t)(-(v + 1)) + 1 : (uint64_t)v;
    do {
        b[n++] = (char)('0' + u % 10);
        u /= 10;
    } while (u);
    if (neg) s += '-';
    while (n) s += b[--n];
}

struct Out {
    FILE* f;
    std::string s;
    explicit Out(FILE* file) : f(file) {}
    void flush_if_big()
    {
        if (s.size() > (1u << 20)) flush();
    }
    void flush()
    {
        fwrite(s.data(), 1, s.size(), f);
        s.clear();
    }
};

int fail(const std::string& msg)
{
    fprintf(stderr, "qc_convert: %s\n", msg.c_str());
    return 1;
}

// the integers of one line (ASCII whitespace separated); false on a token
// that is not a non-negative decimal integer
bool line_ints(const char* p, const char* e, std::vector<int64_t>& v)
{
    v.clear();
    while (p < e) {
        while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\f' || *p == '\v')) p++;
        if (p == e) break;
        if (*p < '0' || *p > '9') return false;
        int64_t x = 0;
        while (p < e && *p >= '0' && *p <= '9') {
            x = x * 10 + (*p - '0');
            if (x > INT32_MAX) return false;
            p++;
        }
        if (p < e && !(*p == ' ' || *p == '\t' || *p == '\r' || *p == '\f' || *p == '\v')) return false;
        v.push_back(x);
    }
    return true;
}

// Lines as a Python text file iterates them: split at '\n', "\r\n" and '\r',
// no empty last line for a file that ends with a line break.
template <class F>
void for_lines(const std::string& s, F f)
{
    size_t i = 0, n = s.size();
    while (i < n) {
        size_t j = i;
        while (j < n && s[j] != '\n' && s[j] != '\r') j++;
        f(s.data() + i, s.data() + j);
        if (j < n && s[j] == '\r' && j + 1 < n && s[j + 1] == '\n') j++;
        i = j + 1;
    }
}

int edges2adj(const char* in, int duplicate, const char* out)
{
    std::string s;
    if (!read_file(in, s)) return fail(std::string("cannot read ") + in);
    std::vector<std::pair<int32_t, int32_t>> edges;
    std::vector<int64_t> v;
    int64_t line = 0;
    bool bad = false;
    for_lines(s, [&](const char* p, const char* e) {
        line++;
        if (bad) return;
        if (!line_ints(p, e, v) || v.size() != 2) {
            bad = true;
            return;
        }
        edges.push_back({(int32_t)v[0], (int32_t)v[1]});
    });
    if (bad) return fail("line " + std::to_string(line) + " of " + in + " is not two non-negative integers");
    int32_t maxv = 0;
    for (auto& e : edges) maxv = std::max(maxv, std::max(e.first, e.second));
    // rows in insertion order: counting pass, then fill
    std::vector<int64_t> off((size_t)maxv + 2, 0);
    for (auto& e : edges) {
        off[(size_t)e.first + 1]++;
        if (duplicate) off[(size_t)e.second + 1]++;
    }
    for (size_t i = 1; i < off.size(); i++) off[i] += off[i - 1];
    std::vector<int32_t> adj((size_t)off.back());
    std::vector<int64_t> at(off.begin(), off.end() - 1);
    for (auto& e : edges) {
        adj[(size_t)at[(size_t)e.first]++] = e.second;
        if (duplicate) adj[(size_t)at[(size_t)e.second]++] = e.first;
    }
    FILE* f = out ? fopen(out, "wb") : stdout;
    if (!f) return fail(std::string("cannot open ") + out + " for writing");
    Out o(f);
    for (int64_t u = 0; u <= maxv; u++) {
        for (int64_t k = off[(size_t)u]; k < off[(size_t)u + 1]; k++) {
            if (k > off[(size_t)u]) o.s += ' ';
            put_num(o.s, adj[(size_t)k]);
        }
        o.s += '\n';
        o.flush_if_big();
    }
    o.flush();
    if (out) fclose(f);
    return 0;
}

int rmempty(const char* in, const char* out)
{
    std::string s;
    if (!read_file(in, s)) return fail(std::string("cannot read ") + in);
    std::vector<std::vector<int32_t>> rows;
    std::vector<int64_t> v;
    bool bad = false;
    int64_t line = 0;
    for_lines(s, [&](const char* p, const char* e) {
        line++;
        if (bad) return;
        if (!line_ints(p, e, v)) {
            bad = true;
            return;
        }
        rows.emplace_back(v.begin(), v.end());
    });
    if (bad) return fail("line " + std::to_string(line) + " of " + in + " holds a token that is not a non-negative integer");
    std::vector<int64_t> map(rows.size(), -1);
    int64_t kept = 0;
    for (size_t i = 0; i < rows.size(); i++)
        if (!rows[i].empty()) map[i] = kept++;
    FILE* f = fopen(out, "wb");
    if (!f) return fail(std::string("cannot open ") + out + " for writing");
    Out o(f);
    for (size_t i = 0; i < rows.size(); i++) {
        if (rows[i].empty()) continue;
        for (size_t k = 0; k < rows[i].size(); k++) {
            const int64_t x = rows[i][k];
            if (x >= (int64_t)rows.size() || map[(size_t)x] < 0) {
                fclose(f);
                return fail("line " + std::to_string(i + 1) + " names vertex " + std::to_string(x) +
                            ", which has no neighbours (or no line)");
            }
            if (k) o.s += ' ';
            put_num(o.s, map[(size_t)x]);
        }
        o.s += '\n';
        o.flush_if_big();
    }
    o.flush();
    fclose(f);
    return 0;
}

// The adjacency list as adjToSer's parser reads it (adjToSer.cpp:60-110): a
// ' ' ends a number (also an empty one, which reads as 0), a '\n' ends a
// vertex (its pending number counts when a digit was seen on the line), a
// '\0' ends the text, and the text's end ends one more vertex.  Rows sorted
// ascending, repeats kept.
int parse_adj(const char* in, int32_t& n, std::vector<int64_t>& off, std::vector<int32_t>& adj)
{
    std::string s;
    if (!read_file(in, s)) return fail(std::string("cannot read ") + in);
    off.assign(1, 0);
    adj.clear();
    int64_t cur = 0;
    bool empty = true;
    for (size_t i = 0; i < s.size(); i++) {
        const char c = s[i];
        if (c == '\n') {
            if (!empty) adj.push_back((int32_t)cur);
            off.push_back((int64_t)adj.size());
            cur = 0;
            empty = true;
        } else if (c == ' ') {
            adj.push_back((int32_t)cur);
            cur = 0;
        } else if (c == '\0') {
            break;
        } else if (c >= '0' && c <= '9') {
            cur = cur * 10 + (c - '0');
            if (cur > INT32_MAX) return fail(std::string("a number in ") + in + " exceeds 2^31-1");
            empty = false;
        } else {
            return fail(std::string("byte ") + std::to_string(i) + " of " + in +
                        " is neither a digit, ' ' nor '\\n'");
        }
    }
    if (!empty) adj.push_back((int32_t)cur);
    off.push_back((int64_t)adj.size());
    if (off.size() - 1 > (size_t)INT32_MAX) return fail("too many vertices");
    n = (int32_t)(off.size() - 1);
    for (int32_t v = 0; v < n; v++) {
        std::sort(adj.begin() + off[(size_t)v], adj.begin() + off[(size_t)v + 1]);
        for (int64_t k = off[(size_t)v]; k < off[(size_t)v + 1]; k++)
            if (adj[(size_t)k] >= n)
                return fail("vertex " + std::to_string(v) + " names vertex " + std::to_string(adj[(size_t)k]) +
                            ", beyond the " + std::to_string(n) + " vertices of the list");
    }
    return 0;
}

#define CU(x)                                                                              \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) return fail(std::string("CUDA: ") + cudaGetErrorString(e_)); \
    } while (0)

// The two-hop lists N(v) u N(N(v)) minus {v} of the rows as given (a self
// loop keeps v, as adjToSer keeps it), built on the GPU.
int twohop_gpu(int32_t n, const std::vector<int64_t>& off, const std::vector<int32_t>& adj,
               std::vector<int64_t>& off2, std::vector<int32_t>& adj2)
{
    if (n > qc_twohop_noalloc_max_vertices()) {
        // a simple symmetric graph goes through the library's general path
        qc_graph* g = nullptr;
        if (qc_graph_from_csr(n, off.data(), adj.data(), &g) != QC_OK)
            return fail(std::string("graphs above ") + std::to_string(qc_twohop_noalloc_max_vertices()) +
                        " vertices need sorted symmetric rows without repeats or self loops: " +
                        qc_last_error());
        const int64_t m2 = qc_graph_num_twohop(g);
        off2.assign(qc_graph_twohop_offsets(g), qc_graph_twohop_offsets(g) + n + 1);
        adj2.assign(qc_graph_twohop_neighbors(g), qc_graph_twohop_neighbors(g) + m2);
        qc_graph_free(g);
        return 0;
    }
    int64_t *d_off = nullptr, *d_off2 = nullptr;
    int32_t *d_adj = nullptr, *d_adj2 = nullptr;
    const size_t m = adj.size();
    CU(cudaMalloc(&d_off, sizeof(int64_t) * (size_t)(n + 1)));
    CU(cudaMalloc(&d_off2, sizeof(int64_t) * (size_t)(n + 1)));
    CU(cudaMalloc(&d_adj, sizeof(int32_t) * std::max<size_t>(m, 1)));
    CU(cudaMemcpy(d_off, off.data(), sizeof(int64_t) * (size_t)(n + 1), cudaMemcpyHostToDevice));
    if (m) CU(cudaMemcpy(d_adj, adj.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice));
    int64_t total = 0;
    qc_status st = qc_twohop_noalloc(n, d_off, d_adj, d_off2, nullptr, 0, &total, nullptr);
    if (st == QC_OK) {
        CU(cudaMalloc(&d_adj2, sizeof(int32_t) * (size_t)std::max<int64_t>(total, 1)));
        st = qc_twohop_noalloc(n, d_off, d_adj, d_off2, d_adj2, total, &total, nullptr);
    }
    if (st != QC_OK) return fail(std::string("two-hop lists: ") + qc_last_error());
    off2.resize((size_t)n + 1);
    adj2.resize((size_t)total);
    CU(cudaMemcpy(off2.data(), d_off2, sizeof(int64_t) * (size_t)(n + 1), cudaMemcpyDeviceToHost));
    if (total) CU(cudaMemcpy(adj2.data(), d_adj2, sizeof(int32_t) * (size_t)total, cudaMemcpyDeviceToHost));
    cudaFree(d_off);
    cudaFree(d_off2);
    cudaFree(d_adj);
    cudaFree(d_adj2);
    return 0;
}

// adjToSer's output (adjToSer.cpp:159-204): n, 2|E|, the two-hop count, then
// the four arrays, space separated, one line each
int write_ser(const char* path, int32_t n, const std::vector<int64_t>& off, const std::vector<int32_t>& adj,
              const std::vector<int64_t>& off2, const std::vector<int32_t>& adj2)
{
    FILE* f = fopen(path, "wb");
    if (!f) return fail(std::string("cannot open ") + path + " for writing");
    Out o(f);
    put_num(o.s, n);
    o.s += '\n';
    put_num(o.s, (int64_t)adj.size());
    o.s += '\n';
    put_num(o.s, (int64_t)adj2.size());
    o.s += '\n';
    auto row = [&](const auto& a) {
        for (size_t i = 0; i < a.size(); i++) {
            if (i) o.s += ' ';
            put_num(o.s, (int64_t)a[i]);
            o.flush_if_big();
        }
        o.s += '\n';
    };
    row(adj);
    row(off);
    row(adj2);
    row(off2);
    o.flush();
    fclose(f);
    return 0;
}

int write_bin(const char* path, int32_t n, const std::vector<int64_t>& off, const std::vector<int32_t>& adj,
              const std::vector<int64_t>* off2, const std::vector<int32_t>* adj2)
{
    FILE* f = fopen(path, "wb");
    if (!f) return fail(std::string("cannot open ") + path + " for writing");
    const int64_t hdr[3] = {n, (int64_t)adj.size(), off2 ? (int64_t)adj2->size() : -1};
    bool ok = fwrite("QCSRBIN1", 1, 8, f) == 8 && fwrite(hdr, 8, 3, f) == 3 &&
              fwrite(off.data(), 8, off.size(), f) == off.size() &&
              fwrite(adj.data(), 4, adj.size(), f) == adj.size();
    const char zero[8] = {0};
    const size_t pad = (8 - (4 * adj.size()) % 8) % 8;
    ok = ok && fwrite(zero, 1, pad, f) == pad;
    if (off2) {
        ok = ok && fwrite(off2->data(), 8, off2->size(), f) == off2->size() &&
             fwrite(adj2->data(), 4, adj2->size(), f) == adj2->size();
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? 0 : fail(std::string("write to ") + path + " failed");
}

int usage()
{
    fprintf(stderr,
            "Usage: qc_convert edges2adj <edge_file> <0 - normal edges / 1 - duplicate edges> [adj_out]\n"
            "       qc_convert rmempty <adj_in> <adj_out>\n"
            "       qc_convert adj2ser <adj_in> <ser_out>\n"
            "       qc_convert adj2bin <adj_in> <bin_out> [two-hop lists 0/1]\n"
            "       qc_convert ser2bin <ser_in> <bin_out>\n"
            "       qc_convert bin2ser <bin_in> <ser_out>\n");
    return 1;
}

} // namespace

int main(int argc, char* argv[])
{
    if (argc < 2) return usage();
    const std::string cmd = argv[1];
    if (cmd == "edges2adj" && (argc == 4 || argc == 5))
        return edges2adj(argv[2], atoi(argv[3]) == 1, argc == 5 ? argv[4] : nullptr);
    if (cmd == "rmempty" && argc == 4) return rmempty(argv[2], argv[3]);
    if ((cmd == "adj2ser" && argc == 4) || (cmd == "adj2bin" && (argc == 4 || argc == 5))) {
        int32_t n = 0;
        std::vector<int64_t> off, off2;
        std::vector<int32_t> adj, adj2;
        if (parse_adj(argv[2], n, off, adj)) return 1;
        const bool two = cmd == "adj2ser" || argc == 4 || atoi(argv[4]) != 0;
        if (two && twohop_gpu(n, off, adj, off2, adj2)) return 1;
        if (cmd == "adj2ser") return write_ser(argv[3], n, off, adj, off2, adj2);
        return write_bin(argv[3], n, off, adj, two ? &off2 : nullptr, two ? &adj2 : nullptr);
    }
    if ((cmd == "ser2bin" || cmd == "bin2ser") && argc == 4) {
        qc_graph* g = nullptr;
        if (qc_graph_read(argv[2], &g) != QC_OK) return fail(qc_last_error());
        const qc_status st = cmd == "ser2bin" ? qc_graph_write_binary(g, argv[3])
                                              : qc_graph_write_serialized(g, argv[3]);
        qc_graph_free(g);
        return st == QC_OK ? 0 : fail(qc_last_error());
    }
    return usage();
}
