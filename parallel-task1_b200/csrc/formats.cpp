// Graph files of the reference library that this library reads and writes
// besides the edge-list binary (capi.cu): the adjacency-list binary and the
// headerless pair files of the BFS sample.  Host code only; each file is
// read with one bulk fread and parsed in memory.
//
// Reference counterparts:
//   GraphStorageAPI::save_to_adjacency_list_bin_file    include/storage/graph_storage_API.hpp:3-35
//   GraphStorageAPI::load_from_adjacency_list_bin_file  include/storage/graph_storage_API.hpp:69-111
//   read_data_from_file (headerless {int32, int32} pairs) sample/bfs.cpp:84-114
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "trav.h"

namespace trav {
void set_error(const std::string &msg);  // capi.cu: the message trav_last_error() returns
}
using trav::set_error;

namespace {

int io_error(const std::string &msg)
{
    set_error(msg);
    return TRAV_ERR_IO;
}

int bad(const char *msg)
{
    set_error(msg);
    return TRAV_ERR_BAD_ARG;
}

using File = std::unique_ptr<FILE, int (*)(FILE *)>;

// Whole file into memory (one fread); false with the error set when it cannot be read.
bool slurp(const char *path, std::vector<unsigned char> &buf)
{
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_error(std::string("cannot open ") + path);
        return false;
    }
    File guard(f, fclose);
    if (fseek(f, 0, SEEK_END) != 0) {
        set_error(std::string("cannot seek in ") + path);
        return false;
    }
    const long long size = ftell(f);
    if (size < 0 || fseek(f, 0, SEEK_SET) != 0) {
        set_error(std::string("cannot size ") + path);
        return false;
    }
    buf.resize((size_t)size);
    if (size > 0 && fread(buf.data(), 1, (size_t)size, f) != (size_t)size) {
        set_error(std::string("short read in ") + path);
        return false;
    }
    return true;
}

template <class T>
T get(const unsigned char *p)
{
    T x;
    memcpy(&x, p, sizeof(T));
    return x;
}

// The 13-byte header shared by both binary formats: bool directed, int32 V,
// int64 E, written field by field without padding.
constexpr size_t kHeader = 13;
constexpr size_t kVertexRecord = 12;  // Vertex<int>{id, value}, then int32 connection count
constexpr size_t kEdgeRecord = 8;     // {int32 dst, float32 weight}

}  // namespace

extern "C" {

int trav_adj_file_read(const char *path, int32_t *vertices, int64_t *edges, int32_t *directed, int32_t *ids,
                       int32_t *values, int64_t *offsets, int32_t *dst, float *w)
{
    if (!path || !vertices || !edges) return bad("path, vertices and edges must not be NULL");
    std::vector<unsigned char> buf;
    if (!slurp(path, buf)) return TRAV_ERR_IO;
    if (buf.size() < kHeader) return io_error("adjacency-list file shorter than its 13-byte header");
    const int32_t V = get<int32_t>(buf.data() + 1);
    const int64_t E = get<int64_t>(buf.data() + 5);
    if (V < 0 || E < 0) return io_error("adjacency-list header holds a negative vertex or edge count");
    // One pass over the vertex records checks the layout before anything is written out: every record fits,
    // the counts are >= 0, they add up to the header's E and nothing follows the last record.
    size_t at = kHeader;
    int64_t total = 0;
    for (int32_t v = 0; v < V; v++) {
        if (buf.size() - at < kVertexRecord)
            return io_error("adjacency-list file ends inside the record of vertex " + std::to_string(v));
        const int32_t cnt = get<int32_t>(buf.data() + at + 8);
        if (cnt < 0) return io_error("adjacency-list record of vertex " + std::to_string(v) + " has a negative count");
        at += kVertexRecord;
        if ((buf.size() - at) / kEdgeRecord < (size_t)cnt)
            return io_error("adjacency-list file ends inside the edges of vertex " + std::to_string(v));
        at += (size_t)cnt * kEdgeRecord;
        total += cnt;
    }
    if (at != buf.size())
        return io_error("adjacency-list file has " + std::to_string(buf.size() - at) +
                        " bytes after its last vertex record");
    if (total != E)
        return io_error("adjacency-list records hold " + std::to_string(total) + " edges, the header says " +
                        std::to_string(E));
    *vertices = V;
    *edges = E;
    if (directed) *directed = buf[0] ? 1 : 0;
    if (!offsets) return TRAV_OK;
    if (!ids || !values || (E > 0 && (!dst || !w))) return bad("ids, values, dst and w must not be NULL with offsets");
    at = kHeader;
    int64_t e = 0;
    for (int32_t v = 0; v < V; v++) {
        ids[v] = get<int32_t>(buf.data() + at);
        values[v] = get<int32_t>(buf.data() + at + 4);
        const int32_t cnt = get<int32_t>(buf.data() + at + 8);
        at += kVertexRecord;
        offsets[v] = e;
        for (int32_t k = 0; k < cnt; k++, e++, at += kEdgeRecord) {
            dst[e] = get<int32_t>(buf.data() + at);
            w[e] = get<float>(buf.data() + at + 4);
        }
    }
    offsets[V] = e;
    return TRAV_OK;
}

int trav_adj_file_write(const char *path, int32_t directed, int32_t vertices, int64_t edges, const int32_t *ids,
                        const int32_t *values, const int64_t *offsets, const int32_t *dst, const float *w)
{
    if (!path || vertices < 0 || edges < 0 || (vertices > 0 && (!ids || !values || !offsets)) ||
        (edges > 0 && (!dst || !w)))
        return bad("path, counts and arrays must be valid");
    if (vertices > 0 && (offsets[0] != 0 || offsets[vertices] != edges))
        return bad("offsets must run from 0 to edges");
    for (int32_t v = 0; v < vertices; v++)
        if (offsets[v + 1] < offsets[v] || offsets[v + 1] - offsets[v] > INT32_MAX)
            return bad("offsets must not fall, and a row holds at most 2^31 - 1 edges");
    std::vector<unsigned char> buf(kHeader + (size_t)vertices * kVertexRecord + (size_t)edges * kEdgeRecord);
    buf[0] = directed ? 1 : 0;
    memcpy(buf.data() + 1, &vertices, 4);
    memcpy(buf.data() + 5, &edges, 8);
    size_t at = kHeader;
    for (int32_t v = 0; v < vertices; v++) {
        const int32_t cnt = (int32_t)(offsets[v + 1] - offsets[v]);
        memcpy(buf.data() + at, &ids[v], 4);
        memcpy(buf.data() + at + 4, &values[v], 4);
        memcpy(buf.data() + at + 8, &cnt, 4);
        at += kVertexRecord;
        for (int64_t e = offsets[v]; e < offsets[v + 1]; e++, at += kEdgeRecord) {
            memcpy(buf.data() + at, &dst[e], 4);
            memcpy(buf.data() + at + 4, &w[e], 4);
        }
    }
    FILE *f = fopen(path, "wb");
    if (!f) return io_error(std::string("cannot create ") + path);
    File guard(f, fclose);
    if (fwrite(buf.data(), 1, buf.size(), f) != buf.size()) return io_error("write failed");
    return TRAV_OK;
}

int trav_pairs_file_read(const char *path, int32_t vertices_pow, int32_t *vertices, int64_t *edges, int32_t *src,
                         int32_t *dst, float *w)
{
    if (!path || !vertices || !edges) return bad("path, vertices and edges must not be NULL");
    if (vertices_pow < 0 || vertices_pow > 30) return bad("vertices_pow must be in [0, 30]");
    std::vector<unsigned char> buf;
    if (!slurp(path, buf)) return TRAV_ERR_IO;
    // The reference sizes the edge count for weighted records (12 bytes) but reads 8-byte pairs, so it takes
    // the first file_size / 12 pairs of the file; the same count is kept here.
    const int64_t E = (int64_t)(buf.size() / 12);
    *vertices = (int32_t)std::pow(2.0, vertices_pow);
    *edges = E;
    if (!src) return TRAV_OK;
    if (E > 0 && (!dst || !w)) return bad("dst and w must not be NULL when src is given");
    for (int64_t e = 0; e < E; e++) {
        src[e] = get<int32_t>(buf.data() + 8 * e);
        dst[e] = get<int32_t>(buf.data() + 8 * e + 4);
        w[e] = 1.0f;
    }
    return TRAV_OK;
}

}  // extern "C"
