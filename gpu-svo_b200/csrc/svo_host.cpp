// svo_host.cpp -- mesh input and OBJ output for the C ABI.
//
// Compiled with -ffp-contract=off: the reference computes these on the host
// (x86-64, SSE, no FMA), every float operation rounded where it is written.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "svo_device.cuh"
#include "svo_host.h"

namespace {

int fail(int code, const std::string &msg) {
    svo::host::set_error(msg.c_str());
    return code;
}

inline float cmaxf(float a, float b) { return a > b ? a : b; }  // src/CUDAUtil.h:77-80

// Appends "%.6g" of the float widened to double (what std::ostream << float
// prints, src/IO.h:8-10); std::to_chars with a precision is specified to
// format exactly as printf does.
inline char *put_g6(char *p, float f) {
    return std::to_chars(p, p + 48, (double)f, std::chars_format::general, 6).ptr;
}

inline char *put_int(char *p, int v) { return std::to_chars(p, p + 16, v).ptr; }

// write_cube (src/IO.h:23-90): 8 "v" lines then 12 "l" lines; the corners
// are origin + (0|w) per axis, with v4 the origin itself.
inline char *put_cube(char *p, const float o[3], float w, size_t faceBegIdx) {
    const float cx[2] = {o[0] + 0.0f, o[0] + w};
    const float cy[2] = {o[1] + 0.0f, o[1] + w};
    const float cz[2] = {o[2] + 0.0f, o[2] + w};
    // (x bit, y bit, z bit) of v1..v8
    static const int vb[8][3] = {{0, 1, 1}, {0, 0, 1}, {0, 1, 0}, {0, 0, 0},
                                 {1, 0, 0}, {1, 1, 0}, {1, 0, 1}, {1, 1, 1}};
    for (int i = 0; i < 8; ++i) {
        float x = cx[vb[i][0]], y = cy[vb[i][1]], z = cz[vb[i][2]];
        if (i == 3) {
            x = o[0];
            y = o[1];
            z = o[2];
        }
        *p++ = 'v';
        *p++ = ' ';
        p = put_g6(p, x);
        *p++ = ' ';
        p = put_g6(p, y);
        *p++ = ' ';
        p = put_g6(p, z);
        *p++ = '\n';
    }
    static const int ln[12][2] = {{1, 2}, {2, 7}, {7, 8}, {8, 1}, {3, 4}, {4, 5},
                                  {5, 6}, {6, 3}, {3, 1}, {4, 2}, {5, 7}, {6, 8}};
    for (int i = 0; i < 12; ++i) {
        *p++ = 'l';
        *p++ = ' ';
        p = put_int(p, (int)(faceBegIdx + ln[i][0]));  // Eigen::Vector2i: int
        *p++ = ' ';
        p = put_int(p, (int)(faceBegIdx + ln[i][1]));
        *p++ = '\n';
    }
    return p;
}

constexpr size_t kCubeMaxBytes = 8 * (3 + 3 * 16) + 12 * (4 + 2 * 12);

struct CubeSrc {
    const float *origin;  // stride in floats
    size_t stride;
    const float *width;
};

// Formats cubes [0, n) with `threads` workers in rounds, writing in order.
template <class Get>
int write_cubes(int64_t n, Get get, const char *path) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(SVO_ERR_IO, std::string("cannot open ") + path);
    const int nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const int64_t per_thread = 1 << 12;
    std::vector<std::vector<char>> bufs(nth, std::vector<char>(per_thread * kCubeMaxBytes));
    std::vector<size_t> lens(nth);
    int rc = SVO_OK;
    for (int64_t round = 0; round < n; round += per_thread * nth) {
        auto work = [&](int k) {
            const int64_t b = round + k * per_thread, e = std::min(n, b + per_thread);
            char *p = bufs[k].data();
            for (int64_t i = b; i < e; ++i) {
                float o[3], w;
                get(i, o, w);
                p = put_cube(p, o, w, (size_t)i * 8);
            }
            lens[k] = b < e ? (size_t)(p - bufs[k].data()) : 0;
        };
        std::vector<std::thread> pool;
        for (int k = 1; k < nth; ++k) pool.emplace_back(work, k);
        work(0);
        for (auto &t : pool) t.join();
        for (int k = 0; k < nth; ++k)
            if (lens[k] && std::fwrite(bufs[k].data(), 1, lens[k], f) != lens[k]) rc = fail(SVO_ERR_IO, "write failed");
    }
    if (std::fclose(f) != 0 && rc == SVO_OK) rc = fail(SVO_ERR_IO, "close failed");
    return rc;
}

}  // namespace

namespace svo::host {

int write_voxels(const uint64_t *keys, int64_t n, const float origin[3], float width, const char *path) {
    return write_cubes(
        n,
        [&](int64_t i, float o[3], float &w) {
            const uint64_t c = keys[i];
            o[0] = origin[0] + width * (float)compact3(c);
            o[1] = origin[1] + width * (float)compact3(c >> 1);
            o[2] = origin[2] + width * (float)compact3(c >> 2);
            w = width;
        },
        path);
}

}  // namespace svo::host

extern "C" {

void svo_free_host(void *p) { std::free(p); }

// BaseModel::loadOBJ (src/BaseModel.cpp:3-25).  The reference reads with
// istream::getline(buffer, 255) until the eof bit is set; this replays that
// on the whole file: lines up to 254 characters are taken, an unterminated
// last line hits end-of-file and is dropped, and a longer line (on which the
// reference loops forever) is an error.  Each line then goes through the same
// sscanf patterns.  Large files are cut at line starts into chunks parsed by
// separate threads and joined in file order; face indices are absolute, so
// the result does not depend on the cut.
int svo_load_obj(const char *path, float **points, int64_t *n_points, int32_t **tris, int64_t *n_tris) {
    svo::host::TraceRange trace("svo: load OBJ");
    if (!path || !points || !n_points || !tris || !n_tris) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(SVO_ERR_IO, std::string("cannot open ") + path);
    std::string data;
    {
        // one read into a buffer of the file's size (then any remainder, for
        // files whose size is not known up front)
        long len = -1;
        if (std::fseek(f, 0, SEEK_END) == 0) len = std::ftell(f);
        std::rewind(f);
        if (len > 0) {
            data.resize((size_t)len);
            data.resize(std::fread(&data[0], 1, (size_t)len, f));
        }
        char buf[1 << 16];
        size_t k;
        while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) data.append(buf, k);
        std::fclose(f);
    }
    const size_t size = data.size();
    constexpr size_t kMinChunk = 256 << 10;
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nc = std::max<size_t>(1, std::min(hw, size / kMinChunk));
    // chunk c holds the lines that start in [start[c], start[c + 1])
    std::vector<size_t> start(nc + 1, size);
    start[0] = 0;
    for (size_t c = 1; c < nc; ++c) {
        const size_t at = c * (size / nc) - 1;
        const void *nl = std::memchr(data.data() + at, '\n', size - at);
        start[c] = std::max(start[c - 1], nl ? (size_t)((const char *)nl - data.data()) + 1 : size);
    }
    std::vector<std::vector<float>> P(nc);
    std::vector<std::vector<int32_t>> T(nc);
    std::vector<int> err(nc, SVO_OK);
    auto parse = [&](size_t c) {
        try {
            char line[256];
            size_t pos = start[c];
            while (pos < start[c + 1]) {
                const void *nl = std::memchr(data.data() + pos, '\n', size - pos);
                const size_t end = nl ? (size_t)((const char *)nl - data.data()) : size;
                const size_t len = end - pos;
                if (len >= 255) {
                    err[c] = SVO_ERR_PARSE;
                    return;
                }
                if (!nl) break;  // unterminated last line: getline sets eofbit first
                std::memcpy(line, data.data() + pos, len);
                line[len] = '\0';
                pos = end + 1;
                float x, y, z;
                int f0, f0_, f1, f1_, f2, f2_;
                if (line[0] == 'v' && line[1] == ' ') {
                    if (std::sscanf(line, "v %f %f %f", &x, &y, &z) == 3) {
                        P[c].push_back(x);
                        P[c].push_back(y);
                        P[c].push_back(z);
                    }
                } else if (line[0] == 'f' && line[1] == ' ') {
                    if (std::sscanf(line, "f %d//%d %d//%d %d//%d", &f0, &f0_, &f1, &f1_, &f2, &f2_) == 6 ||
                        std::sscanf(line, "f %d/%d %d/%d %d/%d", &f0, &f0_, &f1, &f1_, &f2, &f2_) == 6 ||
                        std::sscanf(line, "f %d %d %d", &f0, &f1, &f2) == 3) {
                        T[c].push_back(f0 - 1);
                        T[c].push_back(f1 - 1);
                        T[c].push_back(f2 - 1);
                    }
                }
            }
        } catch (const std::bad_alloc &) {
            err[c] = SVO_ERR_OUT_OF_MEMORY;
        }
    };
    if (nc == 1) {
        parse(0);
    } else {
        std::vector<std::thread> th;
        th.reserve(nc);
        for (size_t c = 0; c < nc; ++c) th.emplace_back(parse, c);
        for (auto &t : th) t.join();
    }
    for (size_t c = 0; c < nc; ++c) {
        if (err[c] == SVO_ERR_PARSE) return fail(SVO_ERR_PARSE, "line longer than 254 characters");
        if (err[c] != SVO_OK) return fail(err[c], "out of host memory");
    }
    size_t np3 = 0, nt3 = 0;
    for (size_t c = 0; c < nc; ++c) {
        np3 += P[c].size();
        nt3 += T[c].size();
    }
    const int64_t np = (int64_t)np3 / 3;
    for (size_t c = 0; c < nc; ++c)
        for (int32_t v : T[c])
            if (v < 0 || v >= np) return fail(SVO_ERR_PARSE, "face index out of range");
    *points = (float *)std::malloc(std::max<size_t>(1, np3) * sizeof(float));
    *tris = (int32_t *)std::malloc(std::max<size_t>(1, nt3) * sizeof(int32_t));
    if (!*points || !*tris) {
        std::free(*points);
        std::free(*tris);
        return fail(SVO_ERR_OUT_OF_MEMORY, "malloc failed");
    }
    size_t po = 0, to = 0;
    for (size_t c = 0; c < nc; ++c) {
        if (!P[c].empty()) std::memcpy(*points + po, P[c].data(), P[c].size() * sizeof(float));
        if (!T[c].empty()) std::memcpy(*tris + to, T[c].data(), T[c].size() * sizeof(int32_t));
        po += P[c].size();
        to += T[c].size();
    }
    *n_points = np;
    *n_tris = (int64_t)nt3 / 3;
    return SVO_OK;
}

// BaseModel(filename) + createMeshBBCube (src/BaseModel.h:24-49,64-73).
int svo_bbox_cube(const float *pts, int64_t n, svo_aabb *out) {
    if (!pts || !out) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    if (n <= 0) return fail(SVO_ERR_EMPTY, "mesh has no vertices");
    float mn[3] = {pts[0], pts[1], pts[2]}, mx[3] = {pts[0], pts[1], pts[2]};
    for (int64_t k = 0; k < n; ++k)
        for (int a = 0; a < 3; ++a) {
            const float v = pts[3 * k + a];
            if (!std::isfinite(v)) return fail(SVO_ERR_INVALID_ARGUMENT, "non-finite vertex coordinate");
            mn[a] = v < mn[a] ? v : mn[a];
            mx[a] = v > mx[a] ? v : mx[a];
        }
    float len[3], amin[3], amax[3];
    for (int a = 0; a < 3; ++a) {
        len[a] = mx[a] - mn[a];
        amin[a] = mn[a];
        amax[a] = mx[a];
    }
    const float maxlen = cmaxf(len[0], cmaxf(len[1], len[2]));
    for (int a = 0; a < 3; ++a) {
        if (maxlen == len[a]) continue;
        const float delta = maxlen - len[a];
        amin[a] = mn[a] - (delta / 2.0f);
        amax[a] = mx[a] + (delta / 2.0f);
    }
    for (int a = 0; a < 3; ++a) {
        const float eps = (amax[a] - amin[a]) / 10001.0f;
        amin[a] -= eps;
        amax[a] += eps;
        out->min[a] = amin[a];
        out->max[a] = amax[a];
        out->width[a] = amax[a] - amin[a];
    }
    return SVO_OK;
}

int svo_write_voxel_keys(const uint64_t *keys, int64_t n, const float origin[3], float width, const char *path) {
    if ((!keys && n > 0) || !origin || !path) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    return svo::host::write_voxels(keys, n, origin, width, path);
}

int svo_write_tree_nodes(const svo_node *nodes, int64_t n, const char *path) {
    if ((!nodes && n > 0) || !path) return fail(SVO_ERR_INVALID_ARGUMENT, "null argument");
    return write_cubes(
        n,
        [&](int64_t i, float o[3], float &w) {
            o[0] = nodes[i].origin[0];
            o[1] = nodes[i].origin[1];
            o[2] = nodes[i].origin[2];
            w = nodes[i].width;
        },
        path);
}

}  // extern "C"
