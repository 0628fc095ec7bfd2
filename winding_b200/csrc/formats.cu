// Capture formats besides .splat, decoded on the device: the binary .ply that
// training writes, Niantic's .spz and PlayCanvas's .sog (readSplats,
// src/scene/splats.js:60-92).
//
// The host does what the reference's browser does for it -- reading the
// .ply's text header, gunzipping a .spz (the reference's DecompressionStream;
// zlib here) -- and checks everything the reference checks, with its
// messages. The per-splat work (property reads, Math.exp, the colour bytes,
// put()'s covariance, the harmonics as half floats) runs one thread a splat
// on the device, in the reference's double arithmetic (jsmath.cuh, put.cuh).
//   .ply  parsePly   src/scene/splats.js:398-468
//   .spz  parseSpz   src/scene/splats.js:227-303
//   .sog  readSog    src/scene/splats.js:95-200 (images decoded by the caller's
//                    decoder, as the reference's by its decodeImage)
#include "jsmath.cuh"
#include "put.cuh"
#include "wsort.h"
#include "wsort_dev.cuh"
#include "wsort_host.h"

#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <initializer_list>
#include <map>
#include <new>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

namespace wsort {

uint32_t pad_splats(uint32_t n);

namespace {

constexpr double kShC0 = 0.28209479177387814;          // scene/splats.js:40
constexpr uint32_t kShCoefficients[5] = {0, 3, 8, 15, 24};
constexpr double kSpzColourScale = 0.15;              // scene/splats.js:211
constexpr uint32_t kSpzMagic = 0x5053474eu;           // 'NGSP'

// ------------------------------------------------------------- device side

__device__ __forceinline__ unsigned long long ordered64(double d) {
    d = d + 0.0;   // -0 and +0 are one value for the box
    const unsigned long long u = (unsigned long long)__double_as_longlong(d);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

// Where decoded splats go, and the running box (3 ordered minima, 3 maxima)
// and first bad index.
struct Sink {
    float4* centers;
    float2* cov;
    int8_t* sexp;
    uint32_t* sh;       // sh_words a splat, or null
    uint32_t sh_words;
    unsigned long long* box;
    uint32_t* bad;
};

struct Box {
    unsigned long long lo[3], hi[3];
};

// put() (scene/splats.js:335-369) for splat i. Returns false (and records i)
// for a position that is not finite.
__device__ bool put_splat(const Sink& o, Box& box, uint32_t i, double x, double y, double z, uint32_t colour,
                          double sx, double sy, double sz, double qw, double qx, double qy, double qz) {
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
        atomicMin(o.bad, i);
        return false;
    }
    o.centers[i] = make_float4(__double2float_rn(x), __double2float_rn(y), __double2float_rn(z),
                               __uint_as_float(colour));
    float c[6];
    covariance_d(sx, sy, sz, qw, qx, qy, qz, c);
    o.cov[3 * (size_t)i] = make_float2(c[0], c[1]);
    o.cov[3 * (size_t)i + 1] = make_float2(c[2], c[3]);
    o.cov[3 * (size_t)i + 2] = make_float2(c[4], c[5]);
    float m = 0.0f;
    bool finite = true;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        m = fmaxf(m, fabsf(c[k]));
        finite = finite && isfinite(c[k]);
    }
    int e = -100;   // the least e with max |entry| <= 2^e, clamped; 127 when not finite
    if (!finite) {
        e = 127;
    } else if (m > 0.0f) {
        frexpf(m, &e);
        e = e < -100 ? -100 : (e > 127 ? 127 : e);
    }
    o.sexp[i] = (int8_t)e;
    const unsigned long long p[3] = {ordered64(x), ordered64(y), ordered64(z)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        box.lo[k] = min(box.lo[k], p[k]);
        box.hi[k] = max(box.hi[k], p[k]);
    }
    return true;
}

__device__ void finish_box(const Sink& o, Box& box) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            box.lo[k] = min(box.lo[k], __shfl_xor_sync(0xffffffffu, box.lo[k], off));
            box.hi[k] = max(box.hi[k], __shfl_xor_sync(0xffffffffu, box.hi[k], off));
        }
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (box.lo[k] != ~0ull) atomicMin(&o.box[k], box.lo[k]);
            if (box.hi[k] != 0ull) atomicMax(&o.box[3 + k], box.hi[k]);
        }
}

// Packs 3 c half floats (c coefficients, red green blue each) into the
// splat's words, the last half of an odd count zero (putSH, :327-333).
__device__ void put_halves(const Sink& o, uint32_t i, const uint32_t* halves, uint32_t nhalves) {
    for (uint32_t w = 0; w < o.sh_words; ++w) {
        const uint32_t a = 2 * w < nhalves ? halves[2 * w] : 0u;
        const uint32_t b = 2 * w + 1 < nhalves ? halves[2 * w + 1] : 0u;
        o.sh[(size_t)i * o.sh_words + w] = a | (b << 16);
    }
}

// .ply property types (PLY_TYPES, :391-396).
enum PlyType : uint8_t { kNone = 0, kI8, kU8, kI16, kU16, kI32, kU32, kF32, kF64 };

constexpr int kPlyNeeds = 14;   // x y z f_dc_0..2 opacity scale_0..2 rot_0..3
constexpr int kPlyFields = kPlyNeeds + 45;

struct PlyLayout {
    uint32_t stride;
    uint32_t rest;            // f_rest_ properties: 0, 9, 24 or 45
    uint32_t coefficients;    // per channel: rest / 3
    uint8_t type[kPlyFields];
    uint32_t offset[kPlyFields];
};

__device__ __forceinline__ double ply_read(const uint8_t* rec, uint8_t type, uint32_t off) {
    const uint8_t* p = rec + off;
    switch (type) {
        case kI8: return (double)(int8_t)p[0];
        case kU8: return (double)p[0];
        case kI16: return (double)(int16_t)(uint16_t)(p[0] | (p[1] << 8));
        case kU16: return (double)(uint16_t)(p[0] | (p[1] << 8));
        case kI32: return (double)(int32_t)(p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24));
        case kU32: return (double)(uint32_t)(p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24));
        case kF32: return (double)__uint_as_float(p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24));
        case kF64: {
            unsigned long long u = 0;
            for (int k = 7; k >= 0; --k) u = (u << 8) | p[k];
            return __longlong_as_double((long long)u);
        }
        default: return 0.0;
    }
}

// Vertices first .. first + n - 1 of the file, whose records start at data.
__global__ void __launch_bounds__(256) ply_kernel(const uint8_t* __restrict__ data, uint32_t n, uint32_t first,
                                                  PlyLayout L, Sink o) {
    Box box;
    for (int k = 0; k < 3; ++k) {
        box.lo[k] = ~0ull;
        box.hi[k] = 0ull;
    }
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint8_t* rec = data + (size_t)j * L.stride;
        const uint32_t i = first + j;
        double v[kPlyNeeds];
#pragma unroll
        for (int k = 0; k < kPlyNeeds; ++k) v[k] = ply_read(rec, L.type[k], L.offset[k]);
        // byte(0.5 + SH_C0 f_dc), byte(sigmoid(opacity)) (:462-464)
        const uint32_t r = jsmath::js_byte(0.5 + kShC0 * v[3]);
        const uint32_t g = jsmath::js_byte(0.5 + kShC0 * v[4]);
        const uint32_t b = jsmath::js_byte(0.5 + kShC0 * v[5]);
        const uint32_t a = jsmath::js_byte(1.0 / (1.0 + jsmath::exp_js(-v[6])));
        const uint32_t colour = r | (g << 8) | (b << 16) | (a << 24);
        const double sx = jsmath::exp_js(v[7]), sy = jsmath::exp_js(v[8]), sz = jsmath::exp_js(v[9]);
        if (!put_splat(o, box, i, v[0], v[1], v[2], colour, sx, sy, sz, v[10], v[11], v[12], v[13])) continue;
        if (o.sh) {
            // coefficient k: red f_rest_k, green f_rest_(k + c), blue f_rest_(k + 2c) (:465-467)
            uint32_t halves[45];
            const uint32_t c = L.coefficients;
            for (uint32_t k = 0; k < c; ++k)
                for (uint32_t ch = 0; ch < 3; ++ch) {
                    const int f = kPlyNeeds + (int)(k + ch * c);
                    halves[3 * k + ch] = jsmath::signed_half(ply_read(rec, L.type[f], L.offset[f]));
                }
            put_halves(o, i, halves, 3 * c);
        }
    }
    finish_box(o, box);
}

struct SpzLayout {
    uint32_t version, count, degree, file_coefficients;
    uint32_t positions, alphas, colours, scales, rotations, sh;   // byte offsets of each field array
    double fixed;                                                  // 1 / 2^fraction
};

__constant__ float kSpzShFlip[15] = {-1, -1, 1, -1, 1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};   // :213

__global__ void __launch_bounds__(256) spz_kernel(const uint8_t* __restrict__ data, SpzLayout L, Sink o) {
    Box box;
    for (int k = 0; k < 3; ++k) {
        box.lo[k] = ~0ull;
        box.hi[k] = 0ull;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.count; i += gridDim.x * blockDim.x) {
        double pos[3];
        for (int a = 0; a < 3; ++a) {
            if (L.version == 1) {
                const uint8_t* p = data + L.positions + (size_t)i * 6 + a * 2;
                pos[a] = jsmath::from_half(p[0] | (p[1] << 8));
            } else {
                const uint8_t* p = data + L.positions + (size_t)i * 9 + a * 3;
                const int32_t v = (int32_t)((uint32_t)(p[0] | (p[1] << 8) | (p[2] << 16)) << 8) >> 8;
                pos[a] = (double)v * L.fixed;
            }
        }
        // Rotation as x, y, z, w (:262-279).
        double q[4];
        if (L.version < 3) {
            const uint8_t* p = data + L.rotations + (size_t)i * 3;
            for (int a = 0; a < 3; ++a) q[a] = (double)p[a] / 127.5 - 1.0;
            q[3] = sqrt(fmax(0.0, 1.0 - ((q[0] * q[0] + q[1] * q[1]) + q[2] * q[2])));
        } else {
            const uint8_t* p = data + L.rotations + (size_t)i * 4;
            uint32_t packed = p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24);
            const uint32_t largest = packed >> 30;
            double sum = 0.0;
            for (int a = 3; a >= 0; --a) {
                if ((uint32_t)a == largest) continue;
                const uint32_t magnitude = packed & 511u;
                const uint32_t negative = (packed >> 9) & 1u;
                packed >>= 10;
                q[a] = 0.7071067811865476 * (double)magnitude / 511.0 * (negative ? -1.0 : 1.0);
                sum = sum + q[a] * q[a];
            }
            q[largest] = sqrt(fmax(0.0, 1.0 - sum));
        }
        const uint8_t* c = data + L.colours + (size_t)i * 3;
        uint32_t rgb[3];
        for (int k = 0; k < 3; ++k) rgb[k] = jsmath::js_byte(0.5 + kShC0 * (((double)c[k] / 255.0 - 0.5) / kSpzColourScale));
        const uint32_t colour = rgb[0] | (rgb[1] << 8) | (rgb[2] << 16) | ((uint32_t)data[L.alphas + i] << 24);
        const uint8_t* s = data + L.scales + (size_t)i * 3;
        const double sx = jsmath::exp_js((double)s[0] / 16.0 - 10.0);
        const double sy = jsmath::exp_js((double)s[1] / 16.0 - 10.0);
        const double sz = jsmath::exp_js((double)s[2] / 16.0 - 10.0);
        // RUB to RDF: y and z negate, the rotation's y and z too (:290-295).
        if (!put_splat(o, box, i, pos[0], -pos[1], -pos[2], colour, sx, sy, sz, q[3], q[0], -q[1], -q[2])) continue;
        if (o.sh) {
            uint32_t halves[45];
            const uint8_t* h = data + L.sh + (size_t)i * L.file_coefficients * 3;
            const uint32_t nc = L.degree == 1 ? 3u : L.degree == 2 ? 8u : 15u;
            for (uint32_t k = 0; k < nc; ++k)
                for (uint32_t ch = 0; ch < 3; ++ch)
                    halves[3 * k + ch] =
                        jsmath::signed_half(((double)h[k * 3 + ch] - 128.0) / 128.0 * (double)kSpzShFlip[k]);
            put_halves(o, i, halves, 3 * nc);
        }
    }
    finish_box(o, box);
}

// .sog (readSog, scene/splats.js:167-199): images already decoded on the
// host, pixel i of each at bytes 4i .. 4i + 3; the codebooks as numbers.
struct SogLayout {
    uint32_t count, degree, per, palette_width;
    unsigned long long palette_bytes;
    const uint8_t *low, *high, *quats, *scales, *sh0, *labels, *palette;
    const double* books;   // scales' codebook, then sh0's, then shN's: 256 each (NaN: no entry)
    double mins[3], maxs[3];
    double sh_count;       // shN.count as a number
};

__global__ void __launch_bounds__(256) sog_kernel(SogLayout L, Sink o) {
    Box box;
    for (int k = 0; k < 3; ++k) {
        box.lo[k] = ~0ull;
        box.hi[k] = 0ull;
    }
    const double* scale_book = L.books;
    const double* colour_book = L.books + 256;
    const double* sh_book = L.books + 512;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.count; i += gridDim.x * blockDim.x) {
        const size_t o4 = (size_t)i * 4;
        // Positions were stored as sign(x) ln(|x| + 1), 16 bits over the
        // means' range ((maxs - mins) || 1).
        double m[3];
        for (int a = 0; a < 3; ++a) {
            const double v = (double)(L.low[o4 + a] | (L.high[o4 + a] << 8));
            double range = L.maxs[a] - L.mins[a];
            if (!(range != 0.0)) range = 1.0;
            const double t = L.mins[a] + range * v / 65535.0;
            const double e = jsmath::exp_js(fabs(t)) - 1.0;
            m[a] = t < 0 ? -e : e;
        }
        // w x y z less the largest, which the alpha byte (252 + its index)
        // names and unit length gives back; below 252, no rotation.
        double q[4] = {1.0, 0.0, 0.0, 0.0};
        const uint32_t tag = L.quats[o4 + 3];
        if (tag >= 252) {
            const uint32_t largest = tag - 252;
            uint32_t k = 0;
            double sum = 0.0;
            for (uint32_t c = 0; c < 4; ++c) {
                if (c == largest) continue;
                q[c] = (((double)L.quats[o4 + k++] / 255.0) * 2.0 - 1.0) / 1.4142135623730951;
                sum = sum + q[c] * q[c];
            }
            q[largest] = sqrt(fmax(0.0, 1.0 - sum));
        }
        uint32_t colour = (uint32_t)L.sh0[o4 + 3] << 24;
        for (int k = 0; k < 3; ++k) colour |= jsmath::js_byte(0.5 + kShC0 * colour_book[L.sh0[o4 + k]]) << (8 * k);
        const double sx = jsmath::exp_js(scale_book[L.scales[o4]]);
        const double sy = jsmath::exp_js(scale_book[L.scales[o4 + 1]]);
        const double sz = jsmath::exp_js(scale_book[L.scales[o4 + 2]]);
        if (!put_splat(o, box, i, m[0], m[1], m[2], colour, sx, sy, sz, q[0], q[1], q[2], q[3])) continue;
        if (!o.sh) continue;
        // The palette: label / 64 rows of 64 entries, each `per` pixels of
        // red, green and blue codebook indices.
        const double label = (double)(L.labels[o4] | (L.labels[o4 + 1] << 8));
        if (label >= L.sh_count) continue;
        const uint32_t lab = (uint32_t)label;
        const unsigned long long row = (unsigned long long)(lab / 64) * L.palette_width + (lab % 64) * L.per;
        uint32_t halves[45];
        uint32_t nh = 0;
        for (uint32_t k = 0; k < L.per; ++k) {
            const unsigned long long c = (row + k) * 4;
            if (c + 2 >= L.palette_bytes) break;
            for (int ch = 0; ch < 3; ++ch) halves[nh++] = jsmath::signed_half(sh_book[L.palette[c + ch]]);
        }
        put_halves(o, i, halves, nh);
    }
    finish_box(o, box);
}

// --------------------------------------------------------------- host side

std::string js_number(double v) {   // Number -> String (shortest round trip) for the messages
    if (v != v) return "NaN";
    if (std::isinf(v)) return v > 0 ? "Infinity" : "-Infinity";
    char b[40];
    if (v == std::floor(v) && std::fabs(v) < 1e21) {
        std::snprintf(b, sizeof b, "%.0f", v);
        return b;
    }
    for (int p = 1; p <= 17; ++p) {
        std::snprintf(b, sizeof b, "%.*g", p, v);
        if (std::strtod(b, nullptr) == v) break;
    }
    return b;
}

// Number(s) for a header word (StringToNumber): white space around it
// ignored, "" is 0, a decimal literal, 0x / 0o / 0b integers, Infinity;
// anything else NaN.
double js_to_number(const std::string& s, bool present) {
    if (!present) return NAN;
    const size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    if (a == std::string::npos) return 0.0;
    const std::string t = s.substr(a, b - a + 1);
    if (t == "Infinity" || t == "+Infinity") return INFINITY;
    if (t == "-Infinity") return -INFINITY;
    if (t.size() > 2 && t[0] == '0' && std::strchr("xXoObB", t[1])) {
        const int base = (t[1] == 'x' || t[1] == 'X') ? 16 : (t[1] == 'o' || t[1] == 'O') ? 8 : 2;
        double v = 0.0;
        for (size_t k = 2; k < t.size(); ++k) {
            const char ch = t[k];
            int dgt = (ch >= '0' && ch <= '9') ? ch - '0' : (ch >= 'a' && ch <= 'f') ? ch - 'a' + 10
                                                           : (ch >= 'A' && ch <= 'F') ? ch - 'A' + 10 : 99;
            if (dgt >= base) return NAN;
            v = v * base + dgt;
        }
        return v;
    }
    for (char ch : t)
        if (!std::strchr("0123456789+-.eE", ch)) return NAN;
    char* end = nullptr;
    const double v = std::strtod(t.c_str(), &end);
    return end == t.c_str() + t.size() ? v : NAN;
}

std::vector<std::string> words_of(const std::string& line) {   // line.trim().split(/\s+/)
    std::vector<std::string> out;
    std::istringstream in(line);
    std::string w;
    while (in >> w) out.push_back(w);
    if (out.empty()) out.push_back("");
    return out;
}

// A new cloud of n splats with its device arrays, degree's harmonics and
// the decode's reduction words; nullptr and an error set on failure.
ws_cloud* new_cloud(ws_ctx* ctx, uint32_t n, uint32_t degree, unsigned long long** words, int* rc) {
    ws_cloud* c = new (std::nothrow) ws_cloud();
    if (!c) {
        *rc = set_error(ctx, WS_ERR_NOMEM, "ws_cloud: out of host memory");
        return nullptr;
    }
    c->ctx = ctx;
    c->n = n;
    const size_t np = pad_splats(n);
    cudaError_t e;
    if ((e = cudaMalloc(&c->centers, np * sizeof(float4))) != cudaSuccess ||
        (e = cudaMalloc(&c->cov, np * 3 * sizeof(float2))) != cudaSuccess ||
        (e = cudaMalloc(&c->sexp, np)) != cudaSuccess || (e = cudaMalloc(words, 8 * sizeof(unsigned long long))) != cudaSuccess) {
        ws_cloud_free(c);
        *rc = cuda_error(ctx, e, "ws_cloud");
        return nullptr;
    }
    if (degree) {
        const uint32_t per = (kShCoefficients[degree] * 3 + 1) / 2;
        if ((e = cudaMalloc(&c->sh, ((size_t)n * per + 1) * 4)) != cudaSuccess) {
            cudaFree(*words);
            ws_cloud_free(c);
            *rc = cuda_error(ctx, e, "ws_cloud harmonics");
            return nullptr;
        }
        cudaMemsetAsync(c->sh, 0, ((size_t)n * per + 1) * 4, ctx->stream);
        c->sh_degree = degree;
        c->sh_words = per;
    }
    cudaMemsetAsync(c->centers, 0, np * sizeof(float4), ctx->stream);
    cudaMemsetAsync(c->cov, 0, np * 3 * sizeof(float2), ctx->stream);
    cudaMemsetAsync(c->sexp, 0x7f, np, ctx->stream);   // padding: no shortcut
    const unsigned long long init[8] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull, 0xFFFFFFFFull, 0ull};
    cudaMemcpyAsync(*words, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream);
    *rc = WS_OK;
    return c;
}

Sink sink_of(ws_cloud* c, unsigned long long* words) {
    Sink o;
    o.centers = c->centers;
    o.cov = c->cov;
    o.sexp = c->sexp;
    o.sh = c->sh;
    o.sh_words = c->sh_words;
    o.box = words;
    o.bad = reinterpret_cast<uint32_t*>(words + 6);
    return o;
}

double unordered64(unsigned long long o) {
    const unsigned long long u = (o & 0x8000000000000000ull) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
    double d;
    std::memcpy(&d, &u, 8);
    return d;
}

// Waits for the decode, reads the box and the first bad index back and
// finishes the cloud (or frees it with the reference's error).
int finish_cloud(ws_ctx* ctx, ws_cloud* c, unsigned long long* words, cudaError_t e, ws_cloud** out) {
    unsigned long long back[8];
    if (e == cudaSuccess) e = cudaMemcpyAsync(back, words, sizeof(back), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(words);
    if (e != cudaSuccess) {
        ws_cloud_free(c);
        return cuda_error(ctx, e, "ws_cloud decode");
    }
    const uint32_t bad = (uint32_t)(back[6] & 0xFFFFFFFFull);
    if (bad != 0xFFFFFFFFu) {
        ws_cloud_free(c);
        return set_error(ctx, WS_ERR_NAN, "splats: splat %u has a position that is not a number", bad);
    }
    for (int k = 0; k < 3; ++k) {
        c->bmin[k] = unordered64(back[k]);
        c->bmax[k] = unordered64(back[3 + k]);
    }
    c->magic = kCloudMagic;
    c->alive = true;
    *out = c;
    return WS_OK;
}

// Copies `bytes` from src to dst with the host's threads (the copy into pinned
// memory is what bounds a streamed upload).
void parallel_copy(void* dst, const void* src, size_t bytes) {
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t parts = std::min<size_t>(hw ? std::min(hw, 8u) : 4u, std::max<size_t>(1, bytes >> 22));
    if (parts <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const size_t each = (bytes + parts - 1) / parts;
    std::vector<std::thread> team;
    for (size_t k = 1; k < parts; ++k)
        team.emplace_back([=] {
            const size_t lo = k * each, hi = std::min(bytes, lo + each);
            if (lo < hi) std::memcpy(static_cast<char*>(dst) + lo, static_cast<const char*>(src) + lo, hi - lo);
        });
    std::memcpy(dst, src, std::min(bytes, each));
    for (auto& t : team) t.join();
}

// Streams n fixed-size records from host memory to the device, a chunk of
// about 32 MB at a time through the context's two pinned and two device
// buffers: while one chunk crosses PCIe and is decoded (`decode(dev, first,
// count)`, queued on the context's stream), the host copies the next one.
// Returns the first CUDA error; the caller's decode launches are checked.
template <class Decode>
cudaError_t stream_records(ws_ctx* ctx, const uint8_t* src, uint32_t n, size_t stride, Decode decode) {
    constexpr size_t kChunkBytes = 32u << 20;
    const uint32_t per = (uint32_t)std::max<size_t>(1, std::min<size_t>(kChunkBytes / stride, n ? n : 1));
    const size_t chunk = (size_t)per * stride;
    cudaError_t e;
    for (int b = 0; b < 2; ++b) {
        if ((e = ctx->load_h[b].ensure(chunk)) != cudaSuccess || (e = ctx->load_d[b].ensure(chunk)) != cudaSuccess)
            return e;
        if (!ctx->load_done[b] && (e = cudaEventCreateWithFlags(&ctx->load_done[b], cudaEventDisableTiming)) != cudaSuccess)
            return e;
    }
    for (uint32_t first = 0, k = 0; first < n; first += per, ++k) {
        const int b = (int)(k & 1u);
        const uint32_t count = std::min(per, n - first);
        const size_t bytes = (size_t)count * stride;
        if (k >= 2 && (e = cudaEventSynchronize(ctx->load_done[b])) != cudaSuccess) return e;   // buffer b is free
        parallel_copy(ctx->load_h[b].p, src + (size_t)first * stride, bytes);
        if ((e = cudaMemcpyAsync(ctx->load_d[b].p, ctx->load_h[b].p, bytes, cudaMemcpyHostToDevice, ctx->stream)) !=
            cudaSuccess)
            return e;
        decode(static_cast<const uint8_t*>(ctx->load_d[b].p), first, count);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = cudaEventRecord(ctx->load_done[b], ctx->stream)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

uint32_t grid_of(ws_ctx* ctx, uint32_t n) {
    const uint32_t want = (n + 255) / 256;
    const uint32_t cap = (uint32_t)ctx->sms * 8u;
    return want < cap ? (want ? want : 1u) : cap;
}

int load_ply(ws_ctx* ctx, const uint8_t* data, size_t len, ws_cloud** out) {
    static const char* marker = "end_header";
    const size_t ml = std::strlen(marker);
    long end = -1;
    const long lim = (long)std::min<size_t>(len, 65536) - (long)ml;
    for (long i = 0; i < lim; ++i)
        if (std::memcmp(data + i, marker, ml) == 0) {
            end = i + (long)ml;
            break;
        }
    if (end < 0) return set_error(ctx, WS_ERR_FORMAT, "splats: a .ply with no end_header");
    if ((size_t)end < len && data[end] == 0x0d) ++end;
    ++end;   // the newline
    const std::string text(reinterpret_cast<const char*>(data), std::min<size_t>((size_t)end, len));
    std::vector<std::string> lines;
    {
        size_t a = 0;
        while (true) {
            const size_t b = text.find('\n', a);
            std::string line = text.substr(a, b == std::string::npos ? std::string::npos : b - a);
            if (!line.empty() && line.back() == '\r' && b != std::string::npos) line.pop_back();
            lines.push_back(line);
            if (b == std::string::npos) break;
            a = b + 1;
        }
    }
    static const std::map<std::string, std::pair<PlyType, uint32_t>> types = {
        {"char", {kI8, 1}},   {"int8", {kI8, 1}},     {"uchar", {kU8, 1}},  {"uint8", {kU8, 1}},
        {"short", {kI16, 2}}, {"int16", {kI16, 2}},   {"ushort", {kU16, 2}}, {"uint16", {kU16, 2}},
        {"int", {kI32, 4}},   {"int32", {kI32, 4}},   {"uint", {kU32, 4}},  {"uint32", {kU32, 4}},
        {"float", {kF32, 4}}, {"float32", {kF32, 4}}, {"double", {kF64, 8}}, {"float64", {kF64, 8}},
    };
    std::string format = "null";
    bool have_vertices = false;
    double count = 0;
    uint64_t stride = 0;
    std::map<std::string, std::pair<PlyType, uint32_t>> at;   // name -> (type, offset); the last of a name wins
    for (const std::string& line : lines) {
        const std::vector<std::string> w = words_of(line);
        if (w[0] == "format") {
            format = w.size() > 1 ? w[1] : "undefined";
        } else if (w[0] == "element") {
            const std::string kind = w.size() > 1 ? w[1] : "undefined";
            if (!have_vertices && kind == "chunk")
                return set_error(ctx, WS_ERR_FORMAT,
                                 "splats: a compressed .ply (from SuperSplat) is not read; export an uncompressed "
                                 ".ply or a .splat");
            if (!have_vertices && kind != "vertex")
                return set_error(ctx, WS_ERR_FORMAT, "splats: a .ply whose first element is '%s', not 'vertex'",
                                 kind.c_str());
            if (have_vertices) break;   // elements after the splats are not needed
            have_vertices = true;
            count = js_to_number(w.size() > 2 ? w[2] : "", w.size() > 2);
        } else if (w[0] == "property" && have_vertices) {
            const std::string t = w.size() > 1 ? w[1] : "undefined";
            if (t == "list")
                return set_error(ctx, WS_ERR_FORMAT,
                                 "splats: a .ply with list properties on its vertices is not a splat capture");
            const auto it = types.find(t);
            if (it == types.end())
                return set_error(ctx, WS_ERR_FORMAT, "splats: unknown .ply property type '%s'", t.c_str());
            at[w.size() > 2 ? w[2] : "undefined"] = {it->second.first, (uint32_t)stride};
            stride += it->second.second;
        }
    }
    if (!have_vertices) return set_error(ctx, WS_ERR_FORMAT, "splats: a .ply with no vertices");
    if (format != "binary_little_endian")
        return set_error(ctx, WS_ERR_FORMAT, "splats: a .ply in '%s' format; only binary_little_endian is read",
                         format.c_str());
    if (!(count == std::floor(count) && count > 0 && std::isfinite(count)))
        return set_error(ctx, WS_ERR_FORMAT, "splats: a .ply with %s vertices", js_number(count).c_str());
    static const char* needs[kPlyNeeds] = {"x",       "y",       "z",       "f_dc_0", "f_dc_1", "f_dc_2", "opacity",
                                           "scale_0", "scale_1", "scale_2", "rot_0",  "rot_1",  "rot_2",  "rot_3"};
    std::string missing;
    for (const char* name : needs)
        if (!at.count(name)) missing += (missing.empty() ? "" : ", ") + std::string(name);
    if (!missing.empty())
        return set_error(ctx, WS_ERR_FORMAT, "splats: this .ply is not a splat capture: no %s", missing.c_str());
    const double need = count * (double)stride;
    if ((double)end + need > (double)len)
        return set_error(ctx, WS_ERR_FORMAT, "splats: the .ply is cut short: %s vertices need %s bytes, it has %s",
                         js_number(count).c_str(), js_number(need).c_str(), js_number((double)len - end).c_str());
    uint32_t rest = 0;
    while (at.count("f_rest_" + std::to_string(rest))) ++rest;
    int degree = -1;
    for (int d = 0; d < 4; ++d)
        if (rest % 3 == 0 && rest / 3 == kShCoefficients[d]) degree = d;
    if (rest > 0 && degree < 1)
        return set_error(ctx, WS_ERR_FORMAT,
                         "splats: a .ply with %u f_rest_ properties; harmonics of degree 1, 2 or 3 have 9, 24 or 45",
                         rest);
    if (degree < 0) degree = 0;
    if (count > WS_MAX_SPLATS)
        return set_error(ctx, WS_ERR_CAPACITY, "splats: %s splats are more than this device holds in one buffer, %u",
                         js_number(count).c_str(), WS_MAX_SPLATS);
    const uint32_t n = (uint32_t)count;
    PlyLayout L;
    std::memset(&L, 0, sizeof(L));
    L.stride = (uint32_t)stride;
    L.rest = rest;
    L.coefficients = rest / 3;
    for (int k = 0; k < kPlyNeeds; ++k) {
        L.type[k] = at[needs[k]].first;
        L.offset[k] = at[needs[k]].second;
    }
    for (uint32_t k = 0; k < rest; ++k) {
        const auto& p = at["f_rest_" + std::to_string(k)];
        L.type[kPlyNeeds + k] = p.first;
        L.offset[kPlyNeeds + k] = p.second;
    }
    cudaSetDevice(ctx->device);
    unsigned long long* words = nullptr;
    int rc;
    ws_cloud* c = new_cloud(ctx, n, (uint32_t)degree, &words, &rc);
    if (!c) return rc;
    const Sink sink = sink_of(c, words);
    cudaError_t e = stream_records(ctx, data + end, n, stride, [&](const uint8_t* dev, uint32_t first, uint32_t count) {
        ply_kernel<<<grid_of(ctx, count), 256, 0, ctx->stream>>>(dev, count, first, L, sink);
    });
    return finish_cloud(ctx, c, words, e, out);
}

int load_spz(ws_ctx* ctx, const uint8_t* gz, size_t len, ws_cloud** out) {
    // gunzip (the reference's DecompressionStream('gzip'))
    std::vector<uint8_t> data;
    {
        z_stream zs;
        std::memset(&zs, 0, sizeof(zs));
        if (inflateInit2(&zs, 16 + MAX_WBITS) != Z_OK) return set_error(ctx, WS_ERR_NOMEM, "splats: gunzip failed");
        zs.next_in = const_cast<Bytef*>(gz);
        zs.avail_in = (uInt)len;
        int z = Z_OK;
        std::vector<uint8_t> chunk(1 << 20);
        while (z != Z_STREAM_END) {
            zs.next_out = chunk.data();
            zs.avail_out = (uInt)chunk.size();
            z = inflate(&zs, Z_NO_FLUSH);
            if (z != Z_OK && z != Z_STREAM_END) break;
            data.insert(data.end(), chunk.data(), chunk.data() + (chunk.size() - zs.avail_out));
            if (z == Z_OK && zs.avail_in == 0 && zs.avail_out != 0) break;
        }
        inflateEnd(&zs);
        if (z != Z_STREAM_END) return set_error(ctx, WS_ERR_FORMAT, "splats: the gzip stream is damaged or cut short");
    }
    const size_t n8 = data.size();
    auto u32 = [&](size_t o) {
        uint32_t v;
        std::memcpy(&v, data.data() + o, 4);
        return v;
    };
    if (n8 < 16 || u32(0) != kSpzMagic) return set_error(ctx, WS_ERR_FORMAT, "splats: gzipped, but not a .spz");
    SpzLayout L;
    std::memset(&L, 0, sizeof(L));
    L.version = u32(4);
    if (L.version < 1 || L.version > 3)
        return set_error(ctx, WS_ERR_FORMAT, "splats: a .spz of version %u; versions 1 to 3 are read", L.version);
    L.count = u32(8);
    const uint32_t file_degree = data[12];
    const uint32_t fraction = data[13];
    if (file_degree > 4)
        return set_error(ctx, WS_ERR_FORMAT, "splats: a .spz with harmonics of degree %u", file_degree);
    L.degree = file_degree < 3 ? file_degree : 3;
    L.file_coefficients = kShCoefficients[file_degree];
    const uint64_t position_bytes = L.version == 1 ? 6 : 9;
    const uint64_t rotation_bytes = L.version >= 3 ? 4 : 3;
    uint64_t at = 16;
    const uint64_t sizes[6] = {position_bytes, 1, 3, 3, rotation_bytes, (uint64_t)L.file_coefficients * 3};
    uint64_t offs[6];
    for (int k = 0; k < 6; ++k) {
        offs[k] = at;
        at += (uint64_t)L.count * sizes[k];
    }
    if (L.count == 0) return set_error(ctx, WS_ERR_FORMAT, "splats: a .spz with no splats");
    if (at > n8)
        return set_error(ctx, WS_ERR_FORMAT, "splats: the .spz is cut short: %u splats need %llu bytes, it has %zu",
                         L.count, (unsigned long long)at, n8);
    if (L.count > WS_MAX_SPLATS)
        return set_error(ctx, WS_ERR_CAPACITY, "splats: %u splats are more than this device holds in one buffer, %u",
                         L.count, WS_MAX_SPLATS);
    L.positions = (uint32_t)offs[0];
    L.alphas = (uint32_t)offs[1];
    L.colours = (uint32_t)offs[2];
    L.scales = (uint32_t)offs[3];
    L.rotations = (uint32_t)offs[4];
    L.sh = (uint32_t)offs[5];
    if (at > 0xFFFFFFFFull) return set_error(ctx, WS_ERR_CAPACITY, "splats: a .spz of more than 4 GiB");
    L.fixed = 1.0 / (double)(int32_t)(1u << (fraction & 31u));   // 1 / (1 << fraction): JavaScript's int32 shift
    cudaSetDevice(ctx->device);
    void* staging = nullptr;
    cudaError_t e = cudaMalloc(&staging, (size_t)at);
    if (e != cudaSuccess) return cuda_error(ctx, e, "ws_cloud_load");
    if ((e = cudaMemcpyAsync(staging, data.data(), (size_t)at, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) {
        cudaFree(staging);
        return cuda_error(ctx, e, "ws_cloud_load upload");
    }
    unsigned long long* words = nullptr;
    int rc;
    ws_cloud* c = new_cloud(ctx, L.count, L.degree, &words, &rc);
    if (!c) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(staging);
        return rc;
    }
    spz_kernel<<<grid_of(ctx, L.count), 256, 0, ctx->stream>>>(static_cast<const uint8_t*>(staging), L,
                                                                 sink_of(c, words));
    e = cudaGetLastError();
    rc = finish_cloud(ctx, c, words, e, out);
    cudaStreamSynchronize(ctx->stream);   // the host copy of the unpacked bytes is freed on return
    cudaFree(staging);
    return rc;
}

// ------------------------------------------------------------------- .sog
// The container (a zip: unzip, scene/splats.js:95-125), meta.json and the
// checks of readSog (:127-166), with the reference's messages, on the host;
// the caller's decoder plays decodeImage.

// A value JSON.parse gives, or undefined (a property that is not there).
struct Json {
    enum Kind : uint8_t { kUndefined, kNull, kBool, kNumber, kString, kArray, kObject };
    Kind kind = kUndefined;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> items;
    std::vector<std::pair<std::string, Json>> fields;
};

// JSON.parse's grammar (RFC 8259): duplicate keys, the last wins. Nesting
// is limited (a deeper document is refused, as V8 refuses one too deep
// for its stack).
class JsonParser {
  public:
    JsonParser(const char* p, const char* end) : p_(p), end_(end) {}
    bool parse(Json& out) {
        skip();
        if (!value(out, 0)) return false;
        skip();
        return p_ == end_;
    }

  private:
    const char *p_, *end_;
    void skip() {
        while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) ++p_;
    }
    bool literal(const char* w) {
        const size_t n = std::strlen(w);
        if ((size_t)(end_ - p_) < n || std::memcmp(p_, w, n) != 0) return false;
        p_ += n;
        return true;
    }
    static void utf8(std::string& s, uint32_t c) {
        if (c < 0x80) {
            s += (char)c;
        } else if (c < 0x800) {
            s += (char)(0xC0 | (c >> 6));
            s += (char)(0x80 | (c & 63));
        } else if (c < 0x10000) {
            s += (char)(0xE0 | (c >> 12));
            s += (char)(0x80 | ((c >> 6) & 63));
            s += (char)(0x80 | (c & 63));
        } else {
            s += (char)(0xF0 | (c >> 18));
            s += (char)(0x80 | ((c >> 12) & 63));
            s += (char)(0x80 | ((c >> 6) & 63));
            s += (char)(0x80 | (c & 63));
        }
    }
    bool hex4(uint32_t* v) {
        if (end_ - p_ < 4) return false;
        uint32_t x = 0;
        for (int k = 0; k < 4; ++k) {
            const char c = *p_++;
            x <<= 4;
            if (c >= '0' && c <= '9') x |= (uint32_t)(c - '0');
            else if (c >= 'a' && c <= 'f') x |= (uint32_t)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') x |= (uint32_t)(c - 'A' + 10);
            else return false;
        }
        *v = x;
        return true;
    }
    bool string(std::string& s) {
        ++p_;   // the opening quote
        while (p_ < end_) {
            const unsigned char c = (unsigned char)*p_++;
            if (c == '"') return true;
            if (c < 0x20) return false;
            if (c != '\\') {
                s += (char)c;
                continue;
            }
            if (p_ >= end_) return false;
            const char e = *p_++;
            switch (e) {
                case '"': s += '"'; break;
                case '\\': s += '\\'; break;
                case '/': s += '/'; break;
                case 'b': s += '\b'; break;
                case 'f': s += '\f'; break;
                case 'n': s += '\n'; break;
                case 'r': s += '\r'; break;
                case 't': s += '\t'; break;
                case 'u': {
                    uint32_t c1;
                    if (!hex4(&c1)) return false;
                    if (c1 >= 0xD800 && c1 < 0xDC00 && end_ - p_ >= 6 && p_[0] == '\\' && p_[1] == 'u') {
                        const char* back = p_;
                        p_ += 2;
                        uint32_t c2;
                        if (hex4(&c2) && c2 >= 0xDC00 && c2 < 0xE000) {
                            c1 = 0x10000 + ((c1 - 0xD800) << 10) + (c2 - 0xDC00);
                        } else {
                            p_ = back;
                        }
                    }
                    utf8(s, c1);
                    break;
                }
                default: return false;
            }
        }
        return false;
    }
    bool number(double* v) {
        const char* q = p_;
        if (q < end_ && *q == '-') ++q;
        if (q >= end_) return false;
        if (*q == '0') {
            ++q;
        } else if (*q >= '1' && *q <= '9') {
            while (q < end_ && *q >= '0' && *q <= '9') ++q;
        } else {
            return false;
        }
        if (q < end_ && *q == '.') {
            ++q;
            if (q >= end_ || !(*q >= '0' && *q <= '9')) return false;
            while (q < end_ && *q >= '0' && *q <= '9') ++q;
        }
        if (q < end_ && (*q == 'e' || *q == 'E')) {
            ++q;
            if (q < end_ && (*q == '+' || *q == '-')) ++q;
            if (q >= end_ || !(*q >= '0' && *q <= '9')) return false;
            while (q < end_ && *q >= '0' && *q <= '9') ++q;
        }
        *v = std::strtod(std::string(p_, q).c_str(), nullptr);   // correctly rounded
        p_ = q;
        return true;
    }
    bool value(Json& out, int depth) {
        if (depth > 512 || p_ >= end_) return false;
        const char c = *p_;
        if (c == '{') {
            ++p_;
            out.kind = Json::kObject;
            skip();
            if (p_ < end_ && *p_ == '}') {
                ++p_;
                return true;
            }
            for (;;) {
                skip();
                if (p_ >= end_ || *p_ != '"') return false;
                std::string key;
                if (!string(key)) return false;
                skip();
                if (p_ >= end_ || *p_ != ':') return false;
                ++p_;
                skip();
                Json v;
                if (!value(v, depth + 1)) return false;
                bool replaced = false;
                for (auto& f : out.fields)
                    if (f.first == key) {
                        f.second = std::move(v);
                        replaced = true;
                        break;
                    }
                if (!replaced) out.fields.emplace_back(std::move(key), std::move(v));
                skip();
                if (p_ < end_ && *p_ == ',') {
                    ++p_;
                    continue;
                }
                if (p_ < end_ && *p_ == '}') {
                    ++p_;
                    return true;
                }
                return false;
            }
        }
        if (c == '[') {
            ++p_;
            out.kind = Json::kArray;
            skip();
            if (p_ < end_ && *p_ == ']') {
                ++p_;
                return true;
            }
            for (;;) {
                skip();
                Json v;
                if (!value(v, depth + 1)) return false;
                out.items.push_back(std::move(v));
                skip();
                if (p_ < end_ && *p_ == ',') {
                    ++p_;
                    continue;
                }
                if (p_ < end_ && *p_ == ']') {
                    ++p_;
                    return true;
                }
                return false;
            }
        }
        if (c == '"') {
            out.kind = Json::kString;
            return string(out.str);
        }
        if (literal("true")) {
            out.kind = Json::kBool;
            out.b = true;
            return true;
        }
        if (literal("false")) {
            out.kind = Json::kBool;
            return true;
        }
        if (literal("null")) {
            out.kind = Json::kNull;
            return true;
        }
        out.kind = Json::kNumber;
        return number(&out.num);
    }
};

// v == null || v === undefined: reading a property of it throws.
bool js_nullish(const Json& v) { return v.kind == Json::kUndefined || v.kind == Json::kNull; }

// v[key] for a value that is not null or undefined (an index for arrays and
// strings, a name for objects; anything else has no such property).
Json js_get(const Json& v, const std::string& key) {
    if (v.kind == Json::kObject) {
        for (auto it = v.fields.rbegin(); it != v.fields.rend(); ++it)
            if (it->first == key) return it->second;
        return Json();
    }
    if (v.kind == Json::kArray || v.kind == Json::kString) {
        if (key.empty() || key.size() > 9 || key.find_first_not_of("0123456789") != std::string::npos ||
            (key.size() > 1 && key[0] == '0'))
            return Json();
        const size_t k = std::stoul(key);
        if (v.kind == Json::kArray) return k < v.items.size() ? v.items[k] : Json();
        Json c;   // the code unit at k, for the ASCII strings a codebook could hold
        if (k < v.str.size()) {
            c.kind = Json::kString;
            c.str = v.str.substr(k, 1);
        }
        return c;
    }
    return Json();
}

std::string js_string(const Json& v) {   // String(v)
    switch (v.kind) {
        case Json::kUndefined: return "undefined";
        case Json::kNull: return "null";
        case Json::kBool: return v.b ? "true" : "false";
        case Json::kNumber: return js_number(v.num);
        case Json::kString: return v.str;
        case Json::kArray: {   // Array.prototype.join: null and undefined as ""
            std::string s;
            for (size_t k = 0; k < v.items.size(); ++k) {
                if (k) s += ',';
                if (!js_nullish(v.items[k])) s += js_string(v.items[k]);
            }
            return s;
        }
        default: return "[object Object]";
    }
}

double js_value_number(const Json& v) {   // ToNumber(v)
    switch (v.kind) {
        case Json::kUndefined: return std::nan("");
        case Json::kNull: return 0.0;
        case Json::kBool: return v.b ? 1.0 : 0.0;
        case Json::kNumber: return v.num;
        default: return js_to_number(js_string(v), true);
    }
}

bool js_truthy(const Json& v) {
    switch (v.kind) {
        case Json::kUndefined:
        case Json::kNull: return false;
        case Json::kBool: return v.b;
        case Json::kNumber: return !(v.num == 0.0 || v.num != v.num);
        case Json::kString: return !v.str.empty();
        default: return true;
    }
}

std::string strip_bom(std::string s) {   // TextDecoder drops a leading byte-order mark
    if (s.size() >= 3 && (unsigned char)s[0] == 0xEF && (unsigned char)s[1] == 0xBB && (unsigned char)s[2] == 0xBF)
        s.erase(0, 3);
    return s;
}

struct ZipEntry {
    uint16_t method;
    const uint8_t* data;
    uint32_t size;
};

// The zip's entries by name (a later entry of a name replaces an earlier).
int unzip(ws_ctx* ctx, const uint8_t* d, size_t n, std::map<std::string, ZipEntry>& files) {
    auto u16 = [&](size_t o) -> uint32_t { return o + 2 <= n ? (uint32_t)(d[o] | (d[o + 1] << 8)) : 0u; };
    auto u32 = [&](size_t o) -> uint32_t {
        if (o + 4 > n) return 0u;
        uint32_t v;
        std::memcpy(&v, d + o, 4);
        return v;
    };
    // The end record is the last thing in the file, before a comment of at
    // most 65535 bytes.
    long long end = -1;
    if (n >= 22) {
        const long long lo = n >= 22 + 65535 ? (long long)(n - 22 - 65535) : 0;
        for (long long i = (long long)n - 22; i >= lo; --i)
            if (u32((size_t)i) == 0x06054b50u) {
                end = i;
                break;
            }
    }
    if (end < 0) return set_error(ctx, WS_ERR_FORMAT, "splats: a zip with no end record: cut short?");
    size_t at = u32((size_t)end + 16);
    for (uint32_t k = u16((size_t)end + 10); k > 0; --k) {
        if (at + 46 > n || u32(at) != 0x02014b50u)
            return set_error(ctx, WS_ERR_FORMAT, "splats: a zip whose directory is damaged");
        const uint32_t method = u16(at + 10), size = u32(at + 20), name_len = u16(at + 28), local = u32(at + 42);
        const size_t name_end = std::min(n, at + 46 + name_len);
        const std::string name = strip_bom(std::string(reinterpret_cast<const char*>(d) + at + 46,
                                                       reinterpret_cast<const char*>(d) + name_end));
        if (size == 0xFFFFFFFFu || local == 0xFFFFFFFFu)
            return set_error(ctx, WS_ERR_FORMAT, "splats: a zip64 .sog is not read");
        at += 46 + name_len + u16(at + 30) + u16(at + 32);
        if ((size_t)local + 30 > n)
            return set_error(ctx, WS_ERR_FORMAT, "splats: the zip is cut short in %s", name.c_str());
        const size_t start = (size_t)local + 30 + u16((size_t)local + 26) + u16((size_t)local + 28);
        if (start + size > n) return set_error(ctx, WS_ERR_FORMAT, "splats: the zip is cut short in %s", name.c_str());
        if (method != 0 && method != 8)
            return set_error(ctx, WS_ERR_FORMAT, "splats: %s is compressed with method %u; stored and deflate are read",
                             name.c_str(), method);
        files[name] = ZipEntry{(uint16_t)method, d + start, size};
    }
    return WS_OK;
}

// An entry's bytes: stored, or inflated (raw deflate, the reference's
// DecompressionStream('deflate-raw')).
int entry_bytes(ws_ctx* ctx, const std::string& name, const ZipEntry& e, std::vector<uint8_t>& out) {
    out.clear();
    if (e.method == 0) {
        out.assign(e.data, e.data + e.size);
        return WS_OK;
    }
    z_stream zs;
    std::memset(&zs, 0, sizeof(zs));
    if (inflateInit2(&zs, -MAX_WBITS) != Z_OK) return set_error(ctx, WS_ERR_NOMEM, "splats: inflate failed");
    zs.next_in = const_cast<Bytef*>(e.data);
    zs.avail_in = e.size;
    int z = Z_OK;
    std::vector<uint8_t> chunk(1 << 20);
    while (z != Z_STREAM_END) {
        zs.next_out = chunk.data();
        zs.avail_out = (uInt)chunk.size();
        z = inflate(&zs, Z_NO_FLUSH);
        if (z != Z_OK && z != Z_STREAM_END) break;
        out.insert(out.end(), chunk.data(), chunk.data() + (chunk.size() - zs.avail_out));
        if (z == Z_OK && zs.avail_in == 0 && zs.avail_out != 0) break;
    }
    inflateEnd(&zs);
    if (z != Z_STREAM_END)
        return set_error(ctx, WS_ERR_FORMAT, "splats: %s is not a whole deflate stream", name.c_str());
    return WS_OK;
}

int load_sog(ws_ctx* ctx, const uint8_t* bytes, size_t nbytes, ws_decode_image decode, void* user, ws_cloud** out) {
    std::map<std::string, ZipEntry> files;
    int rc;
    if ((rc = unzip(ctx, bytes, nbytes, files))) return rc;
    std::vector<uint8_t> buf;
    auto file = [&](const Json& name) -> int {   // the entry's bytes into buf
        auto it = name.kind == Json::kString ? files.find(name.str) : files.end();
        if (it == files.end())
            return set_error(ctx, WS_ERR_FORMAT, "splats: the .sog has no %s", js_string(name).c_str());
        return entry_bytes(ctx, it->first, it->second, buf);
    };
    Json meta_name;
    meta_name.kind = Json::kString;
    meta_name.str = "meta.json";
    if ((rc = file(meta_name))) return rc;
    const std::string text = strip_bom(std::string(buf.begin(), buf.end()));
    Json meta;
    if (!JsonParser(text.data(), text.data() + text.size()).parse(meta))
        return set_error(ctx, WS_ERR_FORMAT, "splats: the .sog's meta.json is not JSON");
    // meta.a.b...: the error JavaScript's TypeError stands for when a step
    // reads a property of null or undefined.
    auto member = [&](std::initializer_list<const char*> path, Json* v) -> int {
        Json cur = meta;
        std::string shown;
        for (const char* key : path) {
            if (js_nullish(cur))
                return set_error(ctx, WS_ERR_FORMAT, "splats: the .sog's meta.json has no %s", shown.c_str());
            cur = js_get(cur, key);
            shown += shown.empty() ? key : std::string(".") + key;
        }
        *v = std::move(cur);
        return WS_OK;
    };
    if (js_nullish(meta)) return set_error(ctx, WS_ERR_FORMAT, "splats: the .sog's meta.json has no version");
    const Json version = js_get(meta, "version");
    if (!(version.kind == Json::kNumber && version.num == 2.0))
        return set_error(ctx, WS_ERR_FORMAT,
                         "splats: a .sog of version %s; version 2 is read (re-save it with splat-transform)",
                         js_nullish(version) ? "1" : js_string(version).c_str());
    const Json count_v = js_get(meta, "count");
    if (!(count_v.kind == Json::kNumber && std::isfinite(count_v.num) && count_v.num == std::floor(count_v.num) &&
          count_v.num > 0))
        return set_error(ctx, WS_ERR_FORMAT, "splats: a .sog of %s splats", js_string(count_v).c_str());
    if (count_v.num > (double)WS_MAX_SPLATS)
        return set_error(ctx, WS_ERR_CAPACITY, "splats: %s splats are more than this device holds in one buffer, %u",
                         js_string(count_v).c_str(), WS_MAX_SPLATS);
    const uint32_t count = (uint32_t)count_v.num;

    // The five images every .sog has: their names (in the order the
    // reference reads them), that each is there, then each decoded.
    Json names[5];
    if ((rc = member({"means", "files", "0"}, &names[0])) || (rc = member({"means", "files", "1"}, &names[1])) ||
        (rc = member({"quats", "files", "0"}, &names[2])) || (rc = member({"scales", "files", "0"}, &names[3])) ||
        (rc = member({"sh0", "files", "0"}, &names[4])))
        return rc;
    for (const Json& nm : names)
        if (nm.kind != Json::kString || !files.count(nm.str))
            return set_error(ctx, WS_ERR_FORMAT, "splats: the .sog has no %s", js_string(nm).c_str());
    // Decoded pixels kept on the host: count x 4 bytes of each image (labels
    // sixth), then the palette.
    std::vector<uint8_t> pix;
    auto decoded = [&](const Json& name, bool check, uint32_t* width, size_t* nbytes_out) -> int {
        if ((rc = file(name))) return rc;
        ws_image img{0, 0, nullptr};
        if (decode(user, buf.data(), buf.size(), &img) != 0 || (!img.rgba && img.width && img.height))
            return set_error(ctx, WS_ERR_FORMAT, "splats: decodeImage failed on %s", js_string(name).c_str());
        const unsigned long long pixels = (unsigned long long)img.width * img.height;
        if (check && pixels < count)
            return set_error(ctx, WS_ERR_FORMAT, "splats: %s has %llu pixels, for %u splats", js_string(name).c_str(),
                             pixels, count);
        // An image checked against the count is read for its first `count`
        // pixels; the palette for its first 1024 rows, all that 16-bit labels
        // reach (label / 64 < 1024), though its whole length stays the bound
        // the reference's loop checks.
        const unsigned long long keep = check ? (unsigned long long)count
                                              : std::min<unsigned long long>(pixels, 1024ull * img.width);
        const size_t take = (size_t)keep * 4;
        pix.insert(pix.end(), img.rgba, img.rgba + take);
        if (width) *width = img.width;
        if (nbytes_out) *nbytes_out = (size_t)pixels * 4;
        return WS_OK;
    };
    for (const Json& nm : names)
        if ((rc = decoded(nm, true, nullptr, nullptr))) return rc;
    Json shn;
    if ((rc = member({"shN"}, &shn))) return rc;
    Json bands;
    if (js_truthy(shn)) bands = js_get(shn, "bands");
    const std::string key = bands.kind == Json::kString ? bands.str
                            : bands.kind == Json::kNumber ? js_number(bands.num) : std::string();
    const uint32_t degree = key == "1" ? 1u : key == "2" ? 2u : key == "3" ? 3u : 0u;
    const uint32_t per = kShCoefficients[degree];
    uint32_t palette_width = 0;
    size_t palette_bytes = 0;
    if (degree) {
        Json pname, lname;
        if ((rc = member({"shN", "files", "0"}, &pname))) return rc;
        if ((rc = decoded(pname, false, &palette_width, &palette_bytes))) return rc;
        if ((rc = member({"shN", "files", "1"}, &lname))) return rc;
        // labels go sixth: move the palette's bytes behind them
        std::vector<uint8_t> palette(pix.end() - (ptrdiff_t)palette_bytes, pix.end());
        pix.resize(pix.size() - palette_bytes);
        if ((rc = decoded(lname, true, nullptr, nullptr))) return rc;
        pix.insert(pix.end(), palette.begin(), palette.end());
        if (palette_width != 64 * per)
            return set_error(ctx, WS_ERR_FORMAT, "splats: the .sog's harmonic palette is %u wide; %u for degree %s",
                             palette_width, 64 * per, key.c_str());
    }
    // The numbers the loop reads: the means' ranges and the codebooks (an
    // entry past a codebook's end reads as NaN, as undefined does).
    SogLayout L;
    std::memset(&L, 0, sizeof(L));
    auto numbers = [&](std::initializer_list<const char*> path, double* outv, int k) -> int {
        Json v;
        if ((rc = member(path, &v))) return rc;
        if (js_nullish(v)) {
            std::string shown;
            for (const char* p : path) shown += shown.empty() ? p : std::string(".") + p;
            return set_error(ctx, WS_ERR_FORMAT, "splats: the .sog's meta.json has no %s", shown.c_str());
        }
        for (int j = 0; j < k; ++j) outv[j] = js_value_number(js_get(v, std::to_string(j)));
        return WS_OK;
    };
    std::vector<double> books(768, 0.0);
    if ((rc = numbers({"means", "mins"}, L.mins, 3)) || (rc = numbers({"means", "maxs"}, L.maxs, 3)) ||
        (rc = numbers({"sh0", "codebook"}, books.data() + 256, 256)) ||
        (rc = numbers({"scales", "codebook"}, books.data(), 256)))
        return rc;
    if (degree) {
        if ((rc = numbers({"shN", "codebook"}, books.data() + 512, 256))) return rc;
        L.sh_count = js_value_number(js_get(shn, "count"));
    }

    // Up to the device: the pixels, the codebooks, then one thread a splat.
    const size_t img_bytes = (size_t)count * 4;
    const size_t pix_bytes = pix.size();
    const size_t books_at = (pix_bytes + 255) / 256 * 256;
    const size_t total = books_at + books.size() * sizeof(double);
    cudaSetDevice(ctx->device);
    void* staging = nullptr;
    cudaError_t e = cudaMalloc(&staging, total);
    if (e != cudaSuccess) return cuda_error(ctx, e, "ws_cloud_read");
    uint8_t* dev = static_cast<uint8_t*>(staging);
    if ((e = cudaMemcpyAsync(dev, pix.data(), pix_bytes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dev + books_at, books.data(), books.size() * sizeof(double), cudaMemcpyHostToDevice,
                             ctx->stream)) != cudaSuccess) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(staging);
        return cuda_error(ctx, e, "ws_cloud_read upload");
    }
    L.count = count;
    L.degree = degree;
    L.per = per;
    L.palette_width = palette_width;
    L.palette_bytes = palette_bytes;
    L.low = dev;
    L.high = dev + img_bytes;
    L.quats = dev + 2 * img_bytes;
    L.scales = dev + 3 * img_bytes;
    L.sh0 = dev + 4 * img_bytes;
    L.labels = degree ? dev + 5 * img_bytes : dev;
    L.palette = degree ? dev + 6 * img_bytes : dev;
    L.books = reinterpret_cast<const double*>(dev + books_at);
    unsigned long long* words = nullptr;
    ws_cloud* c = new_cloud(ctx, count, degree, &words, &rc);
    if (!c) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(staging);
        return rc;
    }
    sog_kernel<<<grid_of(ctx, count), 256, 0, ctx->stream>>>(L, sink_of(c, words));
    e = cudaGetLastError();
    rc = finish_cloud(ctx, c, words, e, out);
    cudaStreamSynchronize(ctx->stream);   // the host staging is freed on return
    cudaFree(staging);
    return rc;
}

}  // namespace

cudaError_t launch_decode(const void* records, uint32_t n, float4* centers, float2* cov, int8_t* sexp,
                          uint32_t* bounds, uint32_t* bad, int sms, cudaStream_t stream, uint32_t first);

// n .splat records from host memory into a cloud's arrays, through the
// pinned chunks above.
cudaError_t stream_splat_records(ws_ctx* ctx, const uint8_t* src, uint32_t n, float4* centers, float2* cov,
                                 int8_t* sexp, uint32_t* bounds, uint32_t* bad) {
    cudaError_t le = cudaSuccess;
    const cudaError_t e = stream_records(ctx, src, n, 32, [&](const uint8_t* dev, uint32_t first, uint32_t count) {
        const cudaError_t d = launch_decode(dev, count, centers, cov, sexp, bounds, bad, ctx->sms, ctx->stream, first);
        if (le == cudaSuccess) le = d;
    });
    return e != cudaSuccess ? e : le;
}

}  // namespace wsort

using namespace wsort;

static int cloud_load(ws_ctx* ctx, const uint8_t* bytes, size_t nbytes, ws_cloud** out);

// The loaders size host buffers from the bytes they are given: a request the
// host cannot meet is an error, never an exception across the C ABI.
extern "C" int ws_cloud_load(ws_ctx* ctx, const uint8_t* bytes, size_t nbytes, ws_cloud** out) {
    NvtxRange nvtx("ws_cloud_load");
    try {
        return cloud_load(ctx, bytes, nbytes, out);
    } catch (const std::bad_alloc&) {
        return set_error(ctx, WS_ERR_NOMEM, "ws_cloud_load: out of host memory");
    }
}

static int cloud_load(ws_ctx* ctx, const uint8_t* bytes, size_t nbytes, ws_cloud** out) {
    if (!ctx || !out || (!bytes && nbytes)) return set_error(ctx, WS_ERR_ARG, "ws_cloud_load: null argument");
    *out = nullptr;
    const uint8_t* d = bytes;
    if (nbytes >= 4 && d[0] == 0x50 && d[1] == 0x4b && d[2] == 0x03 && d[3] == 0x04)
        return set_error(ctx, WS_ERR_FORMAT, "splats: a .sog needs decodeImage, for its WebP images");
    if (nbytes >= 2 && d[0] == 0x1f && d[1] == 0x8b) return load_spz(ctx, bytes, nbytes, out);
    if (nbytes >= 8 && d[0] == 0x4e && d[1] == 0x47 && d[2] == 0x53 && d[3] == 0x50) {
        uint32_t version;
        std::memcpy(&version, d + 4, 4);
        if (version >= 4)
            return set_error(ctx, WS_ERR_FORMAT,
                             "splats: a .spz of version 4, compressed with zstd, which browsers cannot unpack; "
                             "save it as version 3, or as a .ply or .splat");
    }
    if (nbytes >= 4 && d[0] == 0x70 && d[1] == 0x6c && d[2] == 0x79 && (d[3] == 0x0a || d[3] == 0x0d))
        return load_ply(ctx, bytes, nbytes, out);
    return ws_cloud_from_splat(ctx, bytes, nbytes, out);
}

extern "C" int ws_cloud_read(ws_ctx* ctx, const uint8_t* bytes, size_t nbytes, ws_decode_image decode, void* user,
                             ws_cloud** out) {
    NvtxRange nvtx("ws_cloud_read");
    if (!ctx || !out || (!bytes && nbytes)) return set_error(ctx, WS_ERR_ARG, "ws_cloud_read: null argument");
    *out = nullptr;
    const uint8_t* d = bytes;
    const bool zip = nbytes >= 4 && d[0] == 0x50 && d[1] == 0x4b && d[2] == 0x03 && d[3] == 0x04;
    if (!zip || !decode) return ws_cloud_load(ctx, bytes, nbytes, out);
    cudaSetDevice(ctx->device);
    try {
        return load_sog(ctx, bytes, nbytes, decode, user, out);
    } catch (const std::bad_alloc&) {
        return set_error(ctx, WS_ERR_NOMEM, "ws_cloud_read: out of host memory");
    }
}

extern "C" int ws_cloud_harmonics(const ws_cloud* c, int* degree, uint32_t* words) {
    if (!c || c->magic != kCloudMagic || !degree) return WS_ERR_ARG;
    if (!c->alive) return WS_ERR_UNLOADED;
    *degree = (int)c->sh_degree;
    if (words && c->sh) {
        cudaSetDevice(c->ctx->device);
        if (cudaMemcpy(words, c->sh, (size_t)c->n * c->sh_words * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            return WS_ERR_CUDA;
    }
    return WS_OK;
}
