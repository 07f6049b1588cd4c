// host.cpp -- graph I/O, gamma tables, level-0 root, maximal filter (host side).
#include "host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <thread>

namespace qcb {

// ------------------------------------------------------------------
// serialized graph I/O
// ------------------------------------------------------------------

namespace {

struct Tok {
    const char* p;
    const char* e;
    bool next(int64_t& v)
    {
        while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t' || *p == '\f' ||
                         *p == '\v'))
            p++;
        if (p >= e) return false;
        bool neg = false;
        if (*p == '-' || *p == '+') {
            neg = *p == '-';
            p++;
        }
        if (p >= e || *p < '0' || *p > '9') return false;
        int64_t x = 0;
        while (p < e && *p >= '0' && *p <= '9') x = x * 10 + (*p++ - '0');
        v = neg ? -x : x;
        return true;
    }
};

void put_num(std::string& s, int64_t v)
{
    char b[24];
    int k = snprintf(b, sizeof(b), "%lld", (long long)v);
    s.append(b, (size_t)k);
}

} // namespace

std::string read_serialized(const char* path, HostGraph& g)
{
    FILE* f = fopen(path, "rb");
    if (!f) return std::string("cannot open graph file ") + path;
    std::string buf;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (sz > 0) {
        buf.resize((size_t)sz);
        if (fread(&buf[0], 1, (size_t)sz, f) != (size_t)sz) {
            fclose(f);
            return "short read on graph file";
        }
    }
    fclose(f);
    Tok t{buf.data(), buf.data() + buf.size()};
    int64_t n, m, m2;
    if (!t.next(n) || !t.next(m) || !t.next(m2)) return "missing header (n, 2|E|, #2-hop)";
    if (n < 0 || n > INT32_MAX || m < 0 || m2 < 0) return "bad header values";
    g.n = (int32_t)n;
    g.adj.resize((size_t)m);
    g.off.resize((size_t)n + 1);
    g.adj2.resize((size_t)m2);
    g.off2.resize((size_t)n + 1);
    int64_t v;
    for (int64_t i = 0; i < m; i++) {
        if (!t.next(v)) return "truncated 1-hop neighbour list";
        g.adj[(size_t)i] = (int32_t)v;
    }
    for (int64_t i = 0; i <= n; i++) {
        if (!t.next(v)) return "truncated 1-hop offsets";
        g.off[(size_t)i] = v;
    }
    for (int64_t i = 0; i < m2; i++) {
        if (!t.next(v)) return "truncated 2-hop neighbour list";
        g.adj2[(size_t)i] = (int32_t)v;
    }
    for (int64_t i = 0; i <= n; i++) {
        if (!t.next(v)) return "truncated 2-hop offsets";
        g.off2[(size_t)i] = v;
    }
    return "";
}

std::string write_serialized(const HostGraph& g, const char* path)
{
    FILE* f = fopen(path, "wb");
    if (!f) return std::string("cannot open ") + path + " for writing";
    std::string s;
    auto flush = [&] {
        fwrite(s.data(), 1, s.size(), f);
        s.clear();
    };
    put_num(s, g.n); s += '\n';
    put_num(s, (int64_t)g.adj.size()); s += '\n';
    put_num(s, (int64_t)g.adj2.size()); s += '\n';
    auto row = [&](const auto& a) {
        for (size_t i = 0; i < a.size(); i++) {
            if (i) s += ' ';
            put_num(s, (int64_t)a[i]);
            if (s.size() > (1u << 20)) flush();
        }
        s += '\n';
    };
    row(g.adj);
    row(g.off);
    row(g.adj2);
    row(g.off2);
    flush();
    fclose(f);
    return "";
}

bool is_binary_graph(const char* path)
{
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    char m[8] = {0};
    const bool ok = fread(m, 1, 8, f) == 8 && memcmp(m, kBinaryMagic, 8) == 0;
    fclose(f);
    return ok;
}

std::string read_binary(const char* path, HostGraph& g, bool& has_twohop)
{
    FILE* f = fopen(path, "rb");
    if (!f) return std::string("cannot open graph file ") + path;
    fseek(f, 0, SEEK_END);
    const int64_t size = (int64_t)ftell(f);
    fseek(f, 0, SEEK_SET);
    char m[8];
    int64_t hdr[3];
    if (fread(m, 1, 8, f) != 8 || memcmp(m, kBinaryMagic, 8) != 0 || fread(hdr, 8, 3, f) != 3) {
        fclose(f);
        return "not a binary CSR graph file";
    }
    const int64_t n = hdr[0], nnz = hdr[1], nnz2 = hdr[2];
    if (n < 0 || n > INT32_MAX || nnz < 0 || nnz2 < -1) {
        fclose(f);
        return "bad header values";
    }
    const int64_t pad = (8 - (nnz * 4) % 8) % 8;
    const int64_t want = 32 + 8 * (n + 1) + 4 * nnz + pad +
                         (nnz2 >= 0 ? 8 * (n + 1) + 4 * nnz2 : 0);
    if (size != want) {
        fclose(f);
        return "file size " + std::to_string(size) + " does not match its header (" +
               std::to_string(want) + " bytes expected)";
    }
    g.n = (int32_t)n;
    g.off.resize((size_t)n + 1);
    g.adj.resize((size_t)nnz);
    bool ok = fread(g.off.data(), 8, (size_t)n + 1, f) == (size_t)n + 1 &&
              fread(g.adj.data(), 4, (size_t)nnz, f) == (size_t)nnz;
    if (ok && pad) {
        char z[8];
        ok = fread(z, 1, (size_t)pad, f) == (size_t)pad;
    }
    has_twohop = nnz2 >= 0;
    g.off2.clear();
    g.adj2.clear();
    if (ok && has_twohop) {
        g.off2.resize((size_t)n + 1);
        g.adj2.resize((size_t)nnz2);
        ok = fread(g.off2.data(), 8, (size_t)n + 1, f) == (size_t)n + 1 &&
             fread(g.adj2.data(), 4, (size_t)nnz2, f) == (size_t)nnz2;
    }
    fclose(f);
    if (!ok) return "short read on graph file";
    return "";
}

std::string write_binary(const HostGraph& g, const char* path)
{
    FILE* f = fopen(path, "wb");
    if (!f) return std::string("cannot open ") + path + " for writing";
    const bool two = g.off2.size() == g.off.size();
    const int64_t hdr[3] = {(int64_t)g.n, (int64_t)g.adj.size(),
                            two ? (int64_t)g.adj2.size() : -1};
    const int64_t pad = (8 - ((int64_t)g.adj.size() * 4) % 8) % 8;
    const char z[8] = {0};
    bool ok = fwrite(kBinaryMagic, 1, 8, f) == 8 && fwrite(hdr, 8, 3, f) == 3 &&
              fwrite(g.off.data(), 8, g.off.size(), f) == g.off.size() &&
              fwrite(g.adj.data(), 4, g.adj.size(), f) == g.adj.size() &&
              (pad == 0 || fwrite(z, 1, (size_t)pad, f) == (size_t)pad);
    if (ok && two)
        ok = fwrite(g.off2.data(), 8, g.off2.size(), f) == g.off2.size() &&
             fwrite(g.adj2.data(), 4, g.adj2.size(), f) == g.adj2.size();
    ok = (fclose(f) == 0) && ok;
    return ok ? "" : std::string("short write on ") + path;
}

// Rows of ids: every row strictly ascending (sorted, no duplicates) with its
// ids in [0, n), checked with branch-free passes the compiler vectorises (a
// row's ids are in range when its first and last are); the exact message is
// looked up only for a failing row.
// (built twice, for AVX2 and for any x86-64, and picked when the library
// loads: the sortedness test is one compare per entry over every row)
#if defined(__x86_64__) && defined(__GNUC__)
__attribute__((target_clones("avx2", "default")))
#endif
static std::string check_rows_range(const int64_t* off, const int32_t* adj, int32_t n, int32_t v0,
                                    int32_t v1, bool no_self, const char* what)
{
    for (int32_t v = v0; v < v1; v++) {
        const int64_t a = off[v], b = off[(size_t)v + 1];
        if (b < a) return std::string(what) + " offsets decrease";
        if (a == b) continue;
        const int32_t* r = adj + a;
        const int64_t len = b - a;
        int bad = r[0] < 0 || r[len - 1] >= n;
        for (int64_t i = 1; i < len; i++) bad |= r[i - 1] >= r[i];
        if (no_self)
            for (int64_t i = 0; i < len; i++) bad |= r[i] == v;
        if (!bad) continue;
        for (int64_t i = 0; i < len; i++) {
            if (r[i] < 0 || r[i] >= n) return std::string(what) + " neighbour id out of range";
            if (no_self && r[i] == v) return std::string("self loop in ") + what + " list";
            if (i > 0 && r[i - 1] >= r[i])
                return std::string(what) + " rows must be sorted ascending without duplicates";
        }
    }
    return "";
}

// The rows of vertices [0, n): sorted, without repeats, ids in range (and no
// self loop).  Large arrays are checked by several host threads, each a
// range of vertices; the first failing range's message is returned.
static std::string check_rows(const int64_t* off, const int32_t* adj, int32_t n, bool no_self,
                              const char* what)
{
    // offsets first: every row must lie inside the array before it is read
    for (int32_t v = 0; v < n; v++)
        if (off[(size_t)v + 1] < off[v]) return std::string(what) + " offsets decrease";
    const int64_t entries = n > 0 ? off[n] - off[0] : 0;
    const int par = entries >= (1 << 22) ? (int)std::min<unsigned>(8, std::max(1u, std::thread::hardware_concurrency())) : 1;
    if (par <= 1) return check_rows_range(off, adj, n, 0, n, no_self, what);
    std::vector<std::string> err((size_t)par);
    std::vector<std::thread> th;
    // ranges of about equal entry counts
    int32_t v0 = 0;
    for (int p = 0; p < par; p++) {
        int32_t v1 = n;
        if (p + 1 < par) {
            const int64_t want = off[0] + entries * (p + 1) / par;
            v1 = (int32_t)(std::lower_bound(off, off + n + 1, want) - off);
            v1 = std::max(v0, std::min(v1, n));
        }
        th.emplace_back([&, p, v0, v1] { err[(size_t)p] = check_rows_range(off, adj, n, v0, v1, no_self, what); });
        v0 = v1;
    }
    for (auto& t : th) t.join();
    for (auto& e : err)
        if (!e.empty()) return e;
    return "";
}

std::string validate(const HostGraph& g, bool need_twohop)
{
    const int32_t n = g.n;
    if ((int64_t)g.off.size() != (int64_t)n + 1) return "1-hop offsets must have n+1 entries";
    if (g.off[0] != 0 || g.off[(size_t)n] != (int64_t)g.adj.size())
        return "1-hop offsets must start at 0 and end at 2|E|";
    std::string e = check_rows(g.off.data(), g.adj.data(), n, true, "1-hop");
    if (!e.empty()) return e;
    // symmetry: w in N(v) <=> v in N(w).  Visiting v in ascending order, the
    // entries v of the sorted rows N(w) come up in order too, so one cursor
    // per row checks every edge once; every row must be used up at the end.
    {
        std::vector<int64_t> cur(g.off.begin(), g.off.end() - 1);
        for (int32_t v = 0; v < n; v++) {
            for (int64_t e = g.off[(size_t)v]; e < g.off[(size_t)v + 1]; e++) {
                int32_t w = g.adj[(size_t)e];
                int64_t& c = cur[(size_t)w];
                if (c >= g.off[(size_t)w + 1] || g.adj[(size_t)c] != v)
                    return "graph is not undirected (asymmetric 1-hop rows)";
                c++;
            }
        }
        for (int32_t w = 0; w < n; w++)
            if (cur[(size_t)w] != g.off[(size_t)w + 1])
                return "graph is not undirected (asymmetric 1-hop rows)";
    }
    if (!need_twohop) return "";
    if ((int64_t)g.off2.size() != (int64_t)n + 1) return "2-hop offsets must have n+1 entries";
    if (g.off2[0] != 0 || g.off2[(size_t)n] != (int64_t)g.adj2.size())
        return "2-hop offsets must start at 0 and end at the 2-hop count";
    return check_rows(g.off2.data(), g.adj2.data(), n, false, "2-hop");
}

// ------------------------------------------------------------------
// gamma tables
// ------------------------------------------------------------------

void gamma_tables(double gamma, int n, int min_size, std::vector<int32_t>& md,
                  std::vector<int32_t>& ubt)
{
    int len = std::max(n, min_size) + 3;
    md.assign((size_t)len, 0);
    ubt.assign((size_t)len, 0);
    for (int i = 1; i < len; i++) md[(size_t)i] = (int32_t)std::ceil(gamma * (double)(i - 1));
    for (int d = 0; d < len; d++) ubt[(size_t)d] = (int32_t)std::floor((double)d / gamma);
}

// ------------------------------------------------------------------
// level 0 (main.cu:846-998)
// ------------------------------------------------------------------

void build_root(const HostGraph& g, const int32_t* md, int min_size, std::vector<int32_t>& ids,
                int& cov)
{
    const int32_t n = g.n;
    const int need = md[min_size];
    std::vector<int32_t> label((size_t)n), exdeg((size_t)n), l2((size_t)n);
    std::vector<int32_t> rem, rmv;
    rem.reserve((size_t)n);
    rmv.reserve((size_t)n);
    for (int32_t i = 0; i < n; i++) {
        exdeg[(size_t)i] = (int32_t)(g.off[(size_t)i + 1] - g.off[(size_t)i]);
        l2[(size_t)i] = g.off2.empty() ? 0 : (int32_t)(g.off2[(size_t)i + 1] - g.off2[(size_t)i]);
        if (exdeg[(size_t)i] >= need && l2[(size_t)i] >= min_size - 1) {
            label[(size_t)i] = 0;
            rem.push_back(i);
        } else {
            label[(size_t)i] = -1;
            rmv.push_back(i);
        }
    }
    // recount while fewer than half of the previous candidates survive
    int64_t ncand = n;
    while ((int64_t)rem.size() < ncand / 2) {
        ncand = (int64_t)rem.size();
        for (int32_t u : rem) exdeg[(size_t)u] = 0;
        for (int32_t u : rem)
            for (int64_t e = g.off[(size_t)u]; e < g.off[(size_t)u + 1]; e++) {
                int32_t w = g.adj[(size_t)e];
                if (label[(size_t)w] == 0) exdeg[(size_t)w]++;
            }
        std::vector<int32_t> keep;
        rmv.clear();
        for (int32_t u : rem) {
            if (exdeg[(size_t)u] >= need) keep.push_back(u);
            else {
                label[(size_t)u] = -1;
                rmv.push_back(u);
            }
        }
        rem.swap(keep);
    }
    // cascade the last removals
    for (size_t k = 0; k < rmv.size(); k++) {
        int32_t u = rmv[k];
        for (int64_t e = g.off[(size_t)u]; e < g.off[(size_t)u + 1]; e++) {
            int32_t w = g.adj[(size_t)e];
            if (label[(size_t)w] == 0) {
                if (--exdeg[(size_t)w] < need) {
                    label[(size_t)w] = -1;
                    rmv.push_back(w);
                }
            }
        }
    }
    // cover vertex: first label-0 vertex of maximum exdeg (strictly > 0)
    int32_t best = 0, best_i = 0;
    for (int32_t i = 0; i < n; i++)
        if (label[(size_t)i] == 0 && exdeg[(size_t)i] > best) {
            best = exdeg[(size_t)i];
            best_i = i;
        }
    ids.clear();
    cov = 0;
    std::vector<int32_t> surv;
    for (int32_t i = 0; i < n; i++)
        if (label[(size_t)i] == 0) surv.push_back(i);
    if (surv.empty()) return;
    label[(size_t)best_i] = 3;
    for (int64_t e = g.off[(size_t)best_i]; e < g.off[(size_t)best_i + 1]; e++) {
        int32_t w = g.adj[(size_t)e];
        if (label[(size_t)w] == 0) label[(size_t)w] = 2;
    }
    // Q order: covered (2), candidates (0), cover (3); then exdeg, 2-hop
    // size, id, all descending (indeg is 0 for every root vertex)
    auto rank = [](int32_t l) { return l == 2 ? 0 : (l == 0 ? 1 : 2); };
    std::sort(surv.begin(), surv.end(), [&](int32_t a, int32_t b) {
        int ra = rank(label[(size_t)a]), rb = rank(label[(size_t)b]);
        if (ra != rb) return ra < rb;
        if (exdeg[(size_t)a] != exdeg[(size_t)b]) return exdeg[(size_t)a] > exdeg[(size_t)b];
        if (l2[(size_t)a] != l2[(size_t)b]) return l2[(size_t)a] > l2[(size_t)b];
        return a > b;
    });
    ids = surv;
    for (int32_t u : surv)
        if (label[(size_t)u] == 2) cov++;
}

// ------------------------------------------------------------------
// maximal filter (host)
// ------------------------------------------------------------------

void maximal_sets(const int32_t* flat, int64_t nints, std::vector<int32_t>& out, int64_t& nsets)
{
    struct S {
        int64_t at;
        int32_t len;
    };
    std::vector<S> sets;
    std::vector<int32_t> pool;
    pool.reserve((size_t)nints);
    int32_t maxid = -1;
    for (int64_t p = 0; p < nints;) {
        int32_t k = flat[p];
        S s{(int64_t)pool.size(), k};
        pool.insert(pool.end(), flat + p + 1, flat + p + 1 + k);
        std::sort(pool.begin() + s.at, pool.end());
        if (k > 0) maxid = std::max(maxid, pool.back());
        sets.push_back(s);
        p += 1 + k;
    }
    auto less = [&](const S& a, const S& b) {
        return std::lexicographical_compare(pool.begin() + a.at, pool.begin() + a.at + a.len,
                                            pool.begin() + b.at, pool.begin() + b.at + b.len);
    };
    auto equal = [&](const S& a, const S& b) {
        return a.len == b.len &&
               std::equal(pool.begin() + a.at, pool.begin() + a.at + a.len, pool.begin() + b.at);
    };
    std::sort(sets.begin(), sets.end(), less);
    sets.erase(std::unique(sets.begin(), sets.end(), equal), sets.end());
    // posting lists
    std::vector<int64_t> start((size_t)maxid + 2, 0);
    for (auto& s : sets)
        for (int32_t i = 0; i < s.len; i++) start[(size_t)pool[(size_t)(s.at + i)] + 1]++;
    for (size_t v = 1; v < start.size(); v++) start[v] += start[v - 1];
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    std::vector<int32_t> post((size_t)start.back());
    for (size_t si = 0; si < sets.size(); si++)
        for (int32_t i = 0; i < sets[si].len; i++)
            post[(size_t)fill[(size_t)pool[(size_t)(sets[si].at + i)]]++] = (int32_t)si;
    out.clear();
    nsets = 0;
    for (size_t si = 0; si < sets.size(); si++) {
        const S& s = sets[si];
        bool keep = true;
        if (s.len > 0) {
            int32_t best = pool[(size_t)s.at];
            for (int32_t i = 1; i < s.len; i++) {
                int32_t v = pool[(size_t)(s.at + i)];
                if (start[(size_t)v + 1] - start[(size_t)v] < start[(size_t)best + 1] - start[(size_t)best])
                    best = v;
            }
            for (int64_t e = start[(size_t)best]; e < start[(size_t)best + 1] && keep; e++) {
                const S& t = sets[(size_t)post[(size_t)e]];
                if (t.len <= s.len) continue;
                if (std::includes(pool.begin() + t.at, pool.begin() + t.at + t.len,
                                  pool.begin() + s.at, pool.begin() + s.at + s.len))
                    keep = false;
            }
        }
        if (keep) {
            out.push_back(s.len);
            out.insert(out.end(), pool.begin() + s.at, pool.begin() + s.at + s.len);
            nsets++;
        }
    }
}

// the lines of sets [a, b) of the flat array (a, b at set starts)
static void format_sets(const int32_t* flat, int64_t a, int64_t b, std::string& s)
{
    s.clear();
    s.reserve((size_t)(b - a) * 7);
    for (int64_t p = a; p < b;) {
        const int32_t k = flat[p];
        put_num(s, k);
        s += ' ';
        for (int32_t i = 0; i < k; i++) {
            put_num(s, flat[p + 1 + i]);
            s += ' ';
        }
        s += '\n';
        p += 1 + k;
    }
}

std::string write_result(const int32_t* flat, int64_t nints, const char* path)
{
    // chunks of about 256 K ints at set boundaries, formatted by up to 16 host
    // threads at a time and written in order
    constexpr int64_t kChunk = 1 << 18;
    std::vector<int64_t> cuts(1, 0);
    for (int64_t p = 0; p < nints;) {
        const int32_t k = flat[p];
        if (k < 0 || p + 1 + k > nints) return "malformed result record";
        p += 1 + k;
        if (p - cuts.back() >= kChunk || p == nints) cuts.push_back(p);
    }
    FILE* f = fopen(path, "wb");
    if (!f) return std::string("cannot open ") + path + " for writing";
    const int64_t nchunks = (int64_t)cuts.size() - 1;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int par = (int)std::min<int64_t>({nchunks, (int64_t)hw, 16});
    std::vector<std::string> bufs((size_t)std::max(par, 1));
    bool ok = true;
    for (int64_t c0 = 0; c0 < nchunks; c0 += std::max(par, 1)) {
        const int64_t c1 = std::min<int64_t>(nchunks, c0 + std::max(par, 1));
        if (c1 - c0 == 1) {
            format_sets(flat, cuts[(size_t)c0], cuts[(size_t)c0 + 1], bufs[0]);
        } else {
            std::vector<std::thread> th;
            for (int64_t c = c0; c < c1; c++)
                th.emplace_back(format_sets, flat, cuts[(size_t)c], cuts[(size_t)c + 1],
                                std::ref(bufs[(size_t)(c - c0)]));
            for (auto& t : th) t.join();
        }
        for (int64_t c = c0; c < c1; c++) {
            const std::string& b = bufs[(size_t)(c - c0)];
            ok = ok && fwrite(b.data(), 1, b.size(), f) == b.size();
        }
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? "" : std::string("write to ") + path + " failed";
}

} // namespace qcb
