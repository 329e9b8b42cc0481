// neurograph's network files straight into a CSR: ngx_network_load and friends (host code only).
//
// Restates the reference's file loading and arc transforms for one process that reads every rank's files:
// FileLoader::load_nodes / load_in_arcs / load_out_arcs (source/graph/FileLoader.cpp:96-327), the per-rank file names
// (make_rank_prefix, FileLoader.cpp:39-48), ArcTransformer::remove_self_arcs / synchronize_arcs / all_weights_one
// (source/graph/ArcTransformer.cpp:21-69) in the order DistributedGraph::construct_graph applies them
// (DistributedGraph.cpp:68-127), and the dropping of zero weights at upload (DistributedGraph.cpp:203-231). Global vertex
// ids are prefix[rank] + local id (AllPairsShortestPath.h:115-117).
//
// Where the reference parses with std::istringstream into per-vertex hash maps on one thread per rank, this parses
// the file bytes directly on all host threads (large files are cut at line boundaries) and merges repeated arcs by a
// counting sort over the source vertex and a sort of each row: the same arcs and summed weights, in target order.

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "ngx_common.cuh"
#include "ngx_network.h"
#include "ngx_threads.h"


namespace ngx {
namespace {

struct RawArc {
    uint32_t u;  // global source
    uint32_t v;  // global target
    int32_t w;
};

std::string rank_prefix(int rank, int number_ranks) {
    const size_t width = std::to_string(number_ranks - 1).size();
    std::string digits = std::to_string(rank);
    return "rank_" + std::string(width > digits.size() ? width - digits.size() : 0, '0') + digits;
}

bool read_file(const std::string& path, std::string& out) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (f == nullptr) {
        return false;
    }
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(size > 0 ? static_cast<size_t>(size) : 0);
    const size_t got = size > 0 ? std::fread(&out[0], 1, out.size(), f) : 0;
    std::fclose(f);
    out.resize(got);
    return true;
}

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// An integer as `istream >> x` reads it within one line: whitespace, an optional sign, at least one digit; stops at
// the first non-digit. Values beyond [lo, hi] fail, as the stream's failbit does.
bool parse_int(const char*& p, const char* end, int64_t lo, int64_t hi, int64_t& out) {
    while (p < end && is_space(*p)) {
        ++p;
    }
    bool neg = false;
    if (p < end && (*p == '+' || *p == '-')) {
        neg = *p == '-';
        ++p;
    }
    if (p >= end || *p < '0' || *p > '9') {
        return false;
    }
    uint64_t v = 0;
    bool overflow = false;
    while (p < end && *p >= '0' && *p <= '9') {
        if (v > (UINT64_MAX - 9) / 10) {
            overflow = true;
        } else {
            v = v * 10 + static_cast<uint64_t>(*p - '0');
        }
        ++p;
    }
    if (overflow || v > static_cast<uint64_t>(INT64_MAX)) {
        return false;
    }
    const int64_t x = neg ? -static_cast<int64_t>(v) : static_cast<int64_t>(v);
    if (x < lo || x > hi) {
        return false;
    }
    out = x;
    return true;
}

// An unsigned 32-bit id as `istream >> uint32_t` reads it: a leading '-' negates modulo 2^32 (so "-1" is 4294967295,
// which no bound accepts).
bool parse_id(const char*& p, const char* end, uint32_t& out) {
    int64_t x = 0;
    if (!parse_int(p, end, -static_cast<int64_t>(UINT32_MAX), UINT32_MAX, x)) {
        return false;
    }
    out = static_cast<uint32_t>(x);
    return true;
}

bool skip_double(const char*& p, const char* end) {
    while (p < end && is_space(*p)) {
        ++p;
    }
    if (p >= end) {
        return false;
    }
    char buf[64];
    const size_t len = std::min<size_t>(static_cast<size_t>(end - p), sizeof(buf) - 1);
    std::memcpy(buf, p, len);
    buf[len] = '\0';
    char* stop = nullptr;
    errno = 0;
    std::strtod(buf, &stop);
    if (stop == buf || errno == ERANGE) {
        return false;
    }
    p += stop - buf;
    return true;
}

bool skip_token(const char*& p, const char* end) {
    while (p < end && is_space(*p)) {
        ++p;
    }
    const char* start = p;
    while (p < end && !is_space(*p)) {
        ++p;
    }
    return p > start;
}

template <typename F>
void for_each_line(const char* begin, const char* end, F&& f) {
    const char* p = begin;
    while (p < end) {
        const char* eol = static_cast<const char*>(std::memchr(p, '\n', static_cast<size_t>(end - p)));
        const char* line_end = eol != nullptr ? eol : end;
        if (line_end > p && *p != '#') {
            f(p, line_end);
        }
        p = eol != nullptr ? eol + 1 : end;
    }
}

// Vertices of one rank: the position lines that parse (id, x, y, z, type) with consecutive 1-based ids
// (FileLoader.cpp:96-176).
int64_t count_nodes(const std::string& text) {
    int64_t count = 0;
    for_each_line(text.data(), text.data() + text.size(), [&](const char* p, const char* e) {
        uint32_t id = 0;
        if (!parse_id(p, e, id) || !skip_double(p, e) || !skip_double(p, e) || !skip_double(p, e) || !skip_token(p, e)) {
            return;
        }
        if (static_cast<int64_t>(id) == count + 1) {
            ++count;
        }
    });
    return count;
}

struct RankInfo {
    const std::vector<int64_t>* nodes;
    const std::vector<int64_t>* prefix;
    int rank;
    int number_ranks;
};

// One network line (FileLoader.cpp:196-249 / 276-326): target rank, target id, source rank, source id, weight and
// an optional plastic flag (0 drops the line). `out` selects the out-arc rules (the source lives on this rank) or
// the in-arc rules (the target does). Returns false for lines the reference skips.
bool parse_arc(const char* p, const char* e, const RankInfo& info, bool out, RawArc& arc) {
    int64_t target_rank = 0, source_rank = 0, weight = 0;
    uint32_t target_id = 0, source_id = 0;
    if (!parse_int(p, e, INT32_MIN, INT32_MAX, target_rank) || !parse_id(p, e, target_id) || !parse_int(p, e, INT32_MIN, INT32_MAX, source_rank) ||
        !parse_id(p, e, source_id) || !parse_int(p, e, INT32_MIN, INT32_MAX, weight)) {
        return false;
    }
    int64_t plastic = 0;
    if (parse_int(p, e, INT32_MIN, INT32_MAX, plastic) && plastic == 0) {
        return false;
    }
    if (weight == 0) {
        return false;
    }
    const std::vector<int64_t>& nodes = *info.nodes;
    const int64_t local_rank = out ? source_rank : target_rank;
    const int64_t other_rank = out ? target_rank : source_rank;
    if (local_rank != info.rank) {
        return false;
    }
    --target_id;  // 1-based in the files
    --source_id;
    const uint32_t local_id = out ? source_id : target_id;
    const uint32_t other_id = out ? target_id : source_id;
    if (static_cast<int64_t>(local_id) >= nodes[static_cast<size_t>(info.rank)]) {
        return false;
    }
    if (other_rank < 0 || other_rank >= info.number_ranks) {
        return false;
    }
    if (static_cast<int64_t>(other_id) >= nodes[static_cast<size_t>(other_rank)]) {
        return false;
    }
    const int64_t local_global = (*info.prefix)[static_cast<size_t>(info.rank)] + local_id;
    const int64_t other_global = (*info.prefix)[static_cast<size_t>(other_rank)] + other_id;
    // out arcs: source -> target; in arcs are kept as target -> source, the direction synchronize_arcs adds them in
    arc.u = static_cast<uint32_t>(local_global);
    arc.v = static_cast<uint32_t>(other_global);
    arc.w = static_cast<int32_t>(weight);
    return true;
}

// Parses `text` with `threads` threads, cutting it at line boundaries.
void parse_arcs(const std::string& text, const RankInfo& info, bool out, int threads, std::vector<std::vector<RawArc>>& parts) {
    const char* begin = text.data();
    const char* end = begin + text.size();
    const int pieces = std::max(1, std::min<int>(threads, static_cast<int>(text.size() / (1 << 20)) + 1));
    std::vector<const char*> cut(static_cast<size_t>(pieces) + 1, end);
    cut[0] = begin;
    for (int i = 1; i < pieces; ++i) {
        const char* c = begin + text.size() * static_cast<size_t>(i) / static_cast<size_t>(pieces);
        c = std::max(c, cut[static_cast<size_t>(i - 1)]);
        const char* nl = static_cast<const char*>(std::memchr(c, '\n', static_cast<size_t>(end - c)));
        cut[static_cast<size_t>(i)] = nl != nullptr ? nl + 1 : end;
    }
    const size_t first = parts.size();
    parts.resize(first + static_cast<size_t>(pieces));
    parallel_for(pieces, pieces, [&](int64_t i) {
        std::vector<RawArc>& mine = parts[first + static_cast<size_t>(i)];
        for_each_line(cut[static_cast<size_t>(i)], cut[static_cast<size_t>(i) + 1], [&](const char* p, const char* e) {
            RawArc arc{};
            if (parse_arc(p, e, info, out, arc)) {
                mine.push_back(arc);
            }
        });
    });
}

// Rows of (target, summed weight) per source, targets ascending and unique; weights summed in 32-bit two's
// complement as the reference's int32 `+=` does.
void merge_rows(int64_t n, const std::vector<std::vector<RawArc>>& parts, int threads, std::vector<int64_t>& row_ptr, std::vector<uint32_t>& col,
                std::vector<int32_t>& w) {
    std::vector<int64_t> count(static_cast<size_t>(n) + 1, 0);
    size_t total = 0;
    for (const auto& part : parts) {
        for (const RawArc& a : part) {
            ++count[a.u + 1];
        }
        total += part.size();
    }
    for (int64_t v = 0; v < n; ++v) {
        count[static_cast<size_t>(v + 1)] += count[static_cast<size_t>(v)];
    }
    std::vector<std::pair<uint32_t, int32_t>> entries(total);
    std::vector<int64_t> fill(count.begin(), count.end() - 1);
    for (const auto& part : parts) {
        for (const RawArc& a : part) {
            entries[static_cast<size_t>(fill[a.u]++)] = { a.v, a.w };
        }
    }
    // sort each row by target, merge repeats (rows split over the threads)
    std::vector<int64_t> kept(static_cast<size_t>(n), 0);
    const int workers = std::max(1, threads);
    parallel_for(workers, workers, [&](int64_t t) {
        for (int64_t v = t; v < n; v += workers) {
            auto* b = entries.data() + count[static_cast<size_t>(v)];
            auto* e = entries.data() + count[static_cast<size_t>(v + 1)];
            std::stable_sort(b, e, [](const auto& x, const auto& y) { return x.first < y.first; });
            int64_t out = 0;
            for (auto* q = b; q < e; ++q) {
                if (out > 0 && b[out - 1].first == q->first) {
                    b[out - 1].second = static_cast<int32_t>(static_cast<uint32_t>(b[out - 1].second) + static_cast<uint32_t>(q->second));
                } else {
                    b[out++] = *q;
                }
            }
            kept[static_cast<size_t>(v)] = out;
        }
    });
    row_ptr.assign(static_cast<size_t>(n) + 1, 0);
    for (int64_t v = 0; v < n; ++v) {
        row_ptr[static_cast<size_t>(v + 1)] = row_ptr[static_cast<size_t>(v)] + kept[static_cast<size_t>(v)];
    }
    col.resize(static_cast<size_t>(row_ptr.back()));
    w.resize(static_cast<size_t>(row_ptr.back()));
    for (int64_t v = 0; v < n; ++v) {
        const auto* b = entries.data() + count[static_cast<size_t>(v)];
        for (int64_t k = 0; k < kept[static_cast<size_t>(v)]; ++k) {
            col[static_cast<size_t>(row_ptr[static_cast<size_t>(v)] + k)] = b[k].first;
            w[static_cast<size_t>(row_ptr[static_cast<size_t>(v)] + k)] = b[k].second;
        }
    }
}

// Removes the arc v -> v from every row.
void erase_self_arcs(int64_t n, std::vector<int64_t>& row_ptr, std::vector<uint32_t>& col, std::vector<int32_t>& w) {
    int64_t out = 0;
    int64_t start = 0;
    for (int64_t v = 0; v < n; ++v) {
        const int64_t end = row_ptr[static_cast<size_t>(v + 1)];
        for (int64_t k = start; k < end; ++k) {
            if (col[static_cast<size_t>(k)] != static_cast<uint32_t>(v)) {
                col[static_cast<size_t>(out)] = col[static_cast<size_t>(k)];
                w[static_cast<size_t>(out)] = w[static_cast<size_t>(k)];
                ++out;
            }
        }
        start = end;
        row_ptr[static_cast<size_t>(v + 1)] = out;
    }
    col.resize(static_cast<size_t>(out));
    w.resize(static_cast<size_t>(out));
}

}  // namespace
}  // namespace ngx

using namespace ngx;

extern "C" {

namespace {
int load_network(const char* directory, int32_t number_ranks, const char* file_prefix, int flags, int threads, ngx_network** out) {
    if (directory == nullptr || out == nullptr || number_ranks < 1) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_network_load: directory or out is NULL, or number_ranks < 1");
    }
    if ((flags & ~(NGX_LOAD_REMOVE_SELF_ARCS | NGX_LOAD_UNDIRECTED | NGX_LOAD_ONE_WEIGHT)) != 0) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_network_load: unknown flags");
    }
    *out = nullptr;
    const int workers = threads > 0 ? threads : std::max(1u, std::thread::hardware_concurrency());
    const std::string dir(directory);
    const std::string prefix = file_prefix != nullptr ? file_prefix : "";
    auto net = std::make_unique<ngx_network>();
    // vertices per rank, then global numbering
    net->rank_nodes.resize(static_cast<size_t>(number_ranks));
    for (int r = 0; r < number_ranks; ++r) {
        std::string text;
        const std::string path = dir + "/positions/" + rank_prefix(r, number_ranks) + "_positions.txt";
        if (!read_file(path, text)) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_network_load: cannot read " + path);
        }
        net->rank_nodes[static_cast<size_t>(r)] = count_nodes(text);
    }
    std::vector<int64_t> rank_prefix_sum(static_cast<size_t>(number_ranks) + 1, 0);
    for (int r = 0; r < number_ranks; ++r) {
        rank_prefix_sum[static_cast<size_t>(r + 1)] = rank_prefix_sum[static_cast<size_t>(r)] + net->rank_nodes[static_cast<size_t>(r)];
    }
    net->n = rank_prefix_sum.back();
    if (net->n >= (int64_t(1) << 31)) {
        return fail(NGX_UNSUPPORTED, "ngx_network_load: more than 2^31 - 1 vertices");
    }
    const bool undirected = (flags & NGX_LOAD_UNDIRECTED) != 0;
    std::vector<std::vector<RawArc>> out_parts, in_parts;
    for (int r = 0; r < number_ranks; ++r) {
        const RankInfo info{ &net->rank_nodes, &rank_prefix_sum, r, number_ranks };
        for (int pass = 0; pass < (undirected ? 2 : 1); ++pass) {
            const bool out_arcs = pass == 0;
            std::string text;
            const std::string path = dir + "/network/" + rank_prefix(r, number_ranks) + prefix + (out_arcs ? "_out_network.txt" : "_in_network.txt");
            if (!read_file(path, text)) {
                return fail(NGX_INVALID_ARGUMENT, "ngx_network_load: cannot read " + path);
            }
            parse_arcs(text, info, out_arcs, workers, out_arcs ? out_parts : in_parts);
        }
    }
    const bool drop_self = (flags & NGX_LOAD_REMOVE_SELF_ARCS) != 0;
    std::vector<int64_t> row_ptr;
    std::vector<uint32_t> col;
    std::vector<int32_t> w;
    merge_rows(net->n, out_parts, workers, row_ptr, col, w);
    out_parts.clear();
    if (drop_self) {
        erase_self_arcs(net->n, row_ptr, col, w);  // ArcTransformer::remove_self_arcs on the out arcs
    }
    if (undirected) {
        // synchronize_arcs: every in arc (t <- s, w) adds w to the out arc t -> s (created at 0); a sum of 0 becomes 1
        std::vector<int64_t> in_row;
        std::vector<uint32_t> in_col;
        std::vector<int32_t> in_w;
        merge_rows(net->n, in_parts, workers, in_row, in_col, in_w);
        in_parts.clear();
        if (drop_self) {
            erase_self_arcs(net->n, in_row, in_col, in_w);  // and on the in arcs
        }
        std::vector<int64_t> m_row(static_cast<size_t>(net->n) + 1, 0);
        std::vector<uint32_t> m_col;
        std::vector<int32_t> m_w;
        m_col.reserve(col.size() + in_col.size());
        m_w.reserve(col.size() + in_col.size());
        for (int64_t v = 0; v < net->n; ++v) {
            int64_t a = row_ptr[static_cast<size_t>(v)];
            const int64_t ae = row_ptr[static_cast<size_t>(v + 1)];
            int64_t b = in_row[static_cast<size_t>(v)];
            const int64_t be = in_row[static_cast<size_t>(v + 1)];
            while (a < ae || b < be) {
                const bool take_a = b >= be || (a < ae && col[static_cast<size_t>(a)] <= in_col[static_cast<size_t>(b)]);
                const bool take_b = a >= ae || (b < be && in_col[static_cast<size_t>(b)] <= col[static_cast<size_t>(a)]);
                const uint32_t target = take_a ? col[static_cast<size_t>(a)] : in_col[static_cast<size_t>(b)];
                int32_t weight = take_a ? w[static_cast<size_t>(a)] : 0;
                if (take_b) {
                    weight = static_cast<int32_t>(static_cast<uint32_t>(weight) + static_cast<uint32_t>(in_w[static_cast<size_t>(b)]));
                    if (weight == 0) {
                        weight = 1;
                    }
                }
                m_col.push_back(target);
                m_w.push_back(weight);
                a += take_a ? 1 : 0;
                b += take_b ? 1 : 0;
            }
            m_row[static_cast<size_t>(v + 1)] = static_cast<int64_t>(m_col.size());
        }
        row_ptr.swap(m_row);
        col.swap(m_col);
        w.swap(m_w);
    }
    if ((flags & NGX_LOAD_ONE_WEIGHT) != 0) {
        // all_weights_one: every stored arc gets weight 1, arcs whose weights summed to 0 included
        std::fill(w.begin(), w.end(), 1);
    }
    // the upload drops zero weights (DistributedGraph.cpp:222-225)
    net->row_ptr.assign(static_cast<size_t>(net->n) + 1, 0);
    net->col.reserve(col.size());
    net->w.reserve(col.size());
    for (int64_t v = 0; v < net->n; ++v) {
        for (int64_t k = row_ptr[static_cast<size_t>(v)]; k < row_ptr[static_cast<size_t>(v + 1)]; ++k) {
            if (w[static_cast<size_t>(k)] != 0) {
                net->col.push_back(static_cast<int32_t>(col[static_cast<size_t>(k)]));
                net->w.push_back(static_cast<double>(w[static_cast<size_t>(k)]));
            }
        }
        net->row_ptr[static_cast<size_t>(v + 1)] = static_cast<int64_t>(net->col.size());
    }
    *out = net.release();
    return NGX_OK;
}
}  // namespace

int ngx_network_load(const char* directory, int32_t number_ranks, const char* file_prefix, int flags, int threads, ngx_network** out) {
    try {
        return load_network(directory, number_ranks, file_prefix, flags, threads, out);
    } catch (const std::bad_alloc&) {
        return fail(NGX_OUT_OF_MEMORY, "ngx_network_load: host allocation failed");
    } catch (const std::exception& e) {
        return fail(NGX_OUT_OF_MEMORY, std::string("ngx_network_load: ") + e.what());
    }
}

int ngx_network_size(const ngx_network* net, int64_t* n, int64_t* m) {
    if (net == nullptr || n == nullptr || m == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_network_size: NULL argument");
    }
    *n = net->n;
    *m = static_cast<int64_t>(net->col.size());
    return NGX_OK;
}

int ngx_network_csr(const ngx_network* net, int64_t* row_ptr, int32_t* col, double* w) {
    if (net == nullptr || row_ptr == nullptr || ((col == nullptr || w == nullptr) && !net->col.empty())) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_network_csr: NULL argument");
    }
    std::memcpy(row_ptr, net->row_ptr.data(), net->row_ptr.size() * sizeof(int64_t));
    if (!net->col.empty()) {
        std::memcpy(col, net->col.data(), net->col.size() * sizeof(int32_t));
        std::memcpy(w, net->w.data(), net->w.size() * sizeof(double));
    }
    return NGX_OK;
}

int ngx_graph_create_from_network(const ngx_network* net, int device, ngx_graph** out) {
    if (net == nullptr || out == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create_from_network: NULL argument");
    }
    ngx_csr csr{};
    csr.n = net->n;
    csr.m = static_cast<int64_t>(net->col.size());
    csr.row_ptr = net->row_ptr.data();
    csr.col = net->col.data();
    csr.w = net->w.data();
    return ngx_graph_create(&csr, device, out);
}

void ngx_network_destroy(ngx_network* net) { delete net; }

}  // extern "C"
