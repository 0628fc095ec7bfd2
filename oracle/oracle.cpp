// CPU oracle for the splat depth-key + stable counting-sort path.
//
// TEST INFRASTRUCTURE ONLY: the checker that tests, the smoke check and the
// benchmark's CPU-baseline leg compare the CUDA library against. Nothing in
// the product library links or calls this file.
//
// Build: g++ -std=c++17 -O2 -ffp-contract=off -fno-fast-math (see Makefile).
// Every f32 operation below is a separately rounded IEEE single op; every
// double operation a separately rounded IEEE double op, evaluated left to
// right as the reference's JavaScript evaluates it.

#include "oracle.h"

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// Math.hypot as V8 evaluates it (the reference's loader runs under V8):
// the largest magnitude is factored out, the squares of the quotients are
// summed with Kahan compensation, and sqrt(sum) * max is returned. Returns
// +0 when every argument is zero (the caller's `|| 1` then applies).
double v8_hypot4(double a, double b, double c, double d) {
    const double v[4] = {std::fabs(a), std::fabs(b), std::fabs(c), std::fabs(d)};
    for (double x : v)   // ECMAScript: an infinite argument wins over NaN
        if (std::isinf(x)) return INFINITY;
    for (double x : v)
        if (std::isnan(x)) return NAN;
    double max = 0.0;
    for (double x : v)
        if (x > max) max = x;
    if (max == 0.0) return 0.0;
    double sum = 0.0, compensation = 0.0;
    for (double x : v) {
        const double n = x / max;
        const double summand = n * n - compensation;
        const double preliminary = sum + summand;
        compensation = (preliminary - sum) - summand;
        sum = preliminary;
    }
    return std::sqrt(sum) * max;
}

float le_f32(const uint8_t* p) {
    float f;
    std::memcpy(&f, p, 4);
    return f;
}

// One decoded splat into the output arrays: put() at scene/splats.js:335-369.
void put(float* centers, float* cov, uint32_t i, const uint8_t* rec) {
    const double x = le_f32(rec + 0), y = le_f32(rec + 4), z = le_f32(rec + 8);
    const double sx = le_f32(rec + 12), sy = le_f32(rec + 16), sz = le_f32(rec + 20);
    centers[size_t(i) * 4 + 0] = static_cast<float>(x);
    centers[size_t(i) * 4 + 1] = static_cast<float>(y);
    centers[size_t(i) * 4 + 2] = static_cast<float>(z);
    const uint32_t word = uint32_t(rec[24]) | (uint32_t(rec[25]) << 8) |
                          (uint32_t(rec[26]) << 16) | (uint32_t(rec[27]) << 24);
    std::memcpy(&centers[size_t(i) * 4 + 3], &word, 4);

    // (b - 128) / 128: exact in double.
    const double qw = (double(rec[28]) - 128.0) / 128.0;
    const double qx = (double(rec[29]) - 128.0) / 128.0;
    const double qy = (double(rec[30]) - 128.0) / 128.0;
    const double qz = (double(rec[31]) - 128.0) / 128.0;
    double length = v8_hypot4(qw, qx, qy, qz);
    if (length == 0.0 || std::isnan(length)) length = 1.0;  // `|| 1`
    const double w = qw / length, u = qx / length, v = qy / length, t = qz / length;
    const double r00 = 1.0 - 2.0 * (v * v + t * t), r01 = 2.0 * (u * v - w * t),
                 r02 = 2.0 * (u * t + w * v);
    const double r10 = 2.0 * (u * v + w * t), r11 = 1.0 - 2.0 * (u * u + t * t),
                 r12 = 2.0 * (v * t - w * u);
    const double r20 = 2.0 * (u * t - w * v), r21 = 2.0 * (v * t + w * u),
                 r22 = 1.0 - 2.0 * (u * u + v * v);
    const double m00 = r00 * sx, m01 = r01 * sy, m02 = r02 * sz;
    const double m10 = r10 * sx, m11 = r11 * sy, m12 = r12 * sz;
    const double m20 = r20 * sx, m21 = r21 * sy, m22 = r22 * sz;
    float* c = cov + size_t(i) * 6;
    c[0] = static_cast<float>(m00 * m00 + m01 * m01 + m02 * m02);
    c[1] = static_cast<float>(m00 * m10 + m01 * m11 + m02 * m12);
    c[2] = static_cast<float>(m00 * m20 + m01 * m21 + m02 * m22);
    c[3] = static_cast<float>(m10 * m10 + m11 * m11 + m12 * m12);
    c[4] = static_cast<float>(m10 * m20 + m11 * m21 + m12 * m22);
    c[5] = static_cast<float>(m20 * m20 + m21 * m21 + m22 * m22);
}

// WGSL clamp(e, low, high) = min(max(e, low), high); max/min return the
// non-NaN operand, as fmaxf/fminf do.
inline float clampf(float e, float lo, float hi) { return std::fmin(std::fmax(e, lo), hi); }

}  // namespace

extern "C" int or_parse_splat(const uint8_t* data, size_t nbytes, float* centers, float* cov,
                              double bmin[3], double bmax[3], uint32_t* bad_index, char* err,
                              size_t errlen) {
    // The sniffing order of parseSplats (scene/splats.js:60-76).
    if (nbytes >= 8 && data[0] == 0x4e && data[1] == 0x47 && data[2] == 0x53 && data[3] == 0x50) {
        uint32_t version;
        std::memcpy(&version, data + 4, 4);
        if (version >= 4) {
            std::snprintf(err, errlen,
                          "splats: a .spz of version 4, compressed with zstd, which browsers cannot "
                          "unpack; save it as version 3, or as a .ply or .splat");
            return -6;
        }
    }
    if (nbytes >= 4 && data[0] == 0x70 && data[1] == 0x6c && data[2] == 0x79 &&
        (data[3] == 0x0a || data[3] == 0x0d)) {
        std::snprintf(err, errlen, "splats: a .ply is not read here: only .splat records are");
        return -5;
    }
    if (nbytes >= 4 && data[0] == 0x50 && data[1] == 0x4b && data[2] == 0x03 && data[3] == 0x04) {
        std::snprintf(err, errlen, "splats: this is a zip: unpack it with readSplats, which reads a .sog");
        return -2;
    }
    if (nbytes >= 2 && data[0] == 0x1f && data[1] == 0x8b) {
        std::snprintf(err, errlen, "splats: this is gzipped: unpack it with readSplats, which reads a .spz");
        return -3;
    }
    if (nbytes == 0 || nbytes % 32 != 0) {
        std::snprintf(err, errlen,
                      "splats: not a .ply, and %zu bytes is not a whole number of 32-byte .splat records",
                      nbytes);
        return -1;
    }
    const uint32_t count = uint32_t(nbytes / 32);
    for (int k = 0; k < 3; ++k) {
        bmin[k] = INFINITY;
        bmax[k] = -INFINITY;
    }
    for (uint32_t i = 0; i < count; ++i) {
        const uint8_t* rec = data + size_t(i) * 32;
        const double p[3] = {le_f32(rec), le_f32(rec + 4), le_f32(rec + 8)};
        if (!(std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]))) {
            if (bad_index) *bad_index = i;
            std::snprintf(err, errlen, "splats: splat %u has a position that is not a number", i);
            return -4;
        }
        put(centers, cov, i, rec);
        for (int k = 0; k < 3; ++k) {
            if (p[k] < bmin[k]) bmin[k] = p[k];
            if (p[k] > bmax[k]) bmax[k] = p[k];
        }
    }
    return 0;
}

extern "C" int or_depth_range(const float mv[16], const double bmin[3], const double bmax[3],
                              float* depth_min, float* depth_scale) {
    // render/splats.js:561-582, in doubles, the box's eight corners.
    double near = INFINITY, far = -INFINITY;
    for (int k = 0; k < 8; ++k) {
        const double x = (k & 1) ? bmax[0] : bmin[0];
        const double y = (k & 2) ? bmax[1] : bmin[1];
        const double z = (k & 4) ? bmax[2] : bmin[2];
        const double depth = -(double(mv[2]) * x + double(mv[6]) * y + double(mv[10]) * z + double(mv[14]));
        if (depth < near) near = depth;
        if (depth > far) far = depth;
    }
    if (far <= 0.0) return 1;
    // Math.max(near, 0): +0 when near is a zero of either sign.
    near = (near > 0.0) ? near : 0.0;
    const double span = far - near;
    *depth_min = static_cast<float>(near);
    *depth_scale = static_cast<float>(65535.0 / (span > 1e-6 ? span : 1e-6));
    return 0;
}

extern "C" void or_footprint(const or_cloud* c, const float* cov, uint32_t i, const float view[4],
                             float f[3]) {
    // render/splats.js:102-124. Matrices are indexed [row][col] here; the
    // WGSL source builds them column by column.
    const float* s6 = cov + size_t(i) * 6;
    const float S[3][3] = {{s6[0], s6[1], s6[2]}, {s6[1], s6[3], s6[4]}, {s6[2], s6[4], s6[5]}};
    const float* P = c->projection;
    const float fx = (P[0] * c->viewport[0]) * 0.5f;
    const float fy = (P[5] * c->viewport[1]) * 0.5f;
    float J[3][3] = {{fx, 0.0f, 0.0f}, {0.0f, fy, 0.0f}, {0.0f, 0.0f, 0.0f}};
    if (P[15] == 0.0f) {
        const float d = -view[2];
        const float x = clampf(view[0] / d, -1.3f / P[0], 1.3f / P[0]) * d;
        const float y = clampf(view[1] / d, -1.3f / P[5], 1.3f / P[5]) * d;
        const float dd = d * d;
        J[0][0] = fx / d;
        J[1][1] = fy / d;
        J[0][2] = (fx * x) / dd;
        J[1][2] = (fy * y) / dd;
    }
    const float* mv = c->model_view;
    float W[3][3];
    for (int r = 0; r < 3; ++r)
        for (int col = 0; col < 3; ++col) W[r][col] = mv[col * 4 + r];
    float T[2][3], U[2][3];
    for (int r = 0; r < 2; ++r)
        for (int col = 0; col < 3; ++col)
            T[r][col] = (J[r][0] * W[0][col] + J[r][1] * W[1][col]) + J[r][2] * W[2][col];
    for (int r = 0; r < 2; ++r)
        for (int col = 0; col < 3; ++col)
            U[r][col] = (T[r][0] * S[0][col] + T[r][1] * S[1][col]) + T[r][2] * S[2][col];
    // cov = U * transpose(T); the WGSL returns cov[0][0], cov[0][1] (column 0,
    // row 1) and cov[1][1].
    f[0] = (U[0][0] * T[0][0] + U[0][1] * T[0][1]) + U[0][2] * T[0][2];
    f[1] = (U[1][0] * T[0][0] + U[1][1] * T[0][1]) + U[1][2] * T[0][2];
    f[2] = (U[1][0] * T[1][0] + U[1][1] * T[1][1]) + U[1][2] * T[1][2];
}

extern "C" uint32_t or_key(const or_cloud* c, const float* centers, const float* cov, uint32_t i) {
    // makeKeys, render/splats.js:155-186.
    const float x = centers[size_t(i) * 4 + 0];
    const float y = centers[size_t(i) * 4 + 1];
    const float z = centers[size_t(i) * 4 + 2];
    uint32_t word;
    std::memcpy(&word, &centers[size_t(i) * 4 + 3], 4);
    const float* M = c->model_view;
    float view[4];
    for (int j = 0; j < 4; ++j) view[j] = ((M[j] * x + M[4 + j] * y) + M[8 + j] * z) + M[12 + j] * 1.0f;
    const float* P = c->projection;
    float clip[4];
    for (int j = 0; j < 4; ++j)
        clip[j] = ((P[j] * view[0] + P[4 + j] * view[1]) + P[8 + j] * view[2]) + P[12 + j] * view[3];
    const float w = clip[3];
    if (view[2] >= 0.0f || clip[2] > w || std::fabs(clip[0]) > 1.3f * w || std::fabs(clip[1]) > 1.3f * w)
        return OR_CULLED;
    // unpack4x8unorm(center.w).a
    const float alpha = float(word >> 24) / 255.0f;
    if (alpha * 255.0f <= 1.0f) return OR_CULLED;
    if (c->cull > 0.0f) {
        float f[3];
        or_footprint(c, cov, i, view, f);
        const float det = (f[0] + 0.3f) * (f[2] + 0.3f) - f[1] * f[1];
        const float area = 6.2831853f * std::sqrt(std::fmax(det, 0.0f));
        if (alpha * area < c->cull) return OR_CULLED;
    }
    const float scaled = (-view[2] - c->depth_min) * c->depth_scale;
    const uint32_t bucket = uint32_t(clampf(scaled, 0.0f, float(OR_BUCKETS - 1u)));
    return OR_BUCKETS - 1u - bucket;
}

extern "C" void or_make_keys(const or_cloud* c, const float* centers, const float* cov, uint32_t begin,
                             uint32_t end, uint32_t* keys) {
    for (uint32_t i = begin; i < end; ++i) keys[i] = or_key(c, centers, cov, i);
}

extern "C" uint32_t or_counting_sort(const uint32_t* keys, uint32_t n, uint32_t* order,
                                     uint32_t* sorted_keys) {
    std::vector<uint32_t> start(OR_BUCKETS + 1, 0);
    for (uint32_t i = 0; i < n; ++i)
        if (keys[i] != OR_CULLED) ++start[keys[i] + 1];
    for (uint32_t b = 0; b < OR_BUCKETS; ++b) start[b + 1] += start[b];
    const uint32_t survivors = start[OR_BUCKETS];
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t k = keys[i];
        if (k == OR_CULLED) continue;
        const uint32_t at = start[k]++;
        order[at] = i;
        if (sorted_keys) sorted_keys[at] = k;
    }
    return survivors;
}

extern "C" void or_drawlist_sort(uint32_t* keys_in, uint32_t* payloads_in, uint32_t n,
                                 uint32_t* keys_alt_in, uint32_t* payloads_alt_in) {
    if (n < 2) return;
    uint32_t* keys = keys_in;
    uint32_t* payloads = payloads_in;
    uint32_t* keys_alt = keys_alt_in;
    uint32_t* payloads_alt = payloads_alt_in;
    uint32_t counts[256];
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = pass * 8;
        std::memset(counts, 0, sizeof(counts));
        for (uint32_t i = 0; i < n; ++i) ++counts[(keys[i] >> shift) & 0xff];
        if (counts[(keys[0] >> shift) & 0xff] == n) continue;
        uint32_t total = 0;
        for (int b = 0; b < 256; ++b) {
            const uint32_t cnt = counts[b];
            counts[b] = total;
            total += cnt;
        }
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t dst = counts[(keys[i] >> shift) & 0xff]++;
            keys_alt[dst] = keys[i];
            payloads_alt[dst] = payloads[i];
        }
        std::swap(keys, keys_alt);
        std::swap(payloads, payloads_alt);
    }
    // The reference repoints its public arrays at whichever pair holds the
    // result; here the result is copied back into the caller's arrays.
    if (keys != keys_in) {
        std::memcpy(keys_in, keys, size_t(n) * 4);
        std::memcpy(payloads_in, payloads, size_t(n) * 4);
    }
}

extern "C" uint32_t or_sort_view(const float* centers, const float* cov, uint32_t n, const double bmin[3],
                                 const double bmax[3], const float model_view[16],
                                 const float projection[16], const float viewport[2], float cull,
                                 uint32_t* order, uint32_t* sorted_keys, int threads) {
    or_cloud c;
    std::memcpy(c.model_view, model_view, sizeof(c.model_view));
    std::memcpy(c.projection, projection, sizeof(c.projection));
    c.viewport[0] = viewport[0];
    c.viewport[1] = viewport[1];
    c.count = n;
    c.cull = cull;
    if (or_depth_range(model_view, bmin, bmax, &c.depth_min, &c.depth_scale) != 0) return 0;
    std::vector<uint32_t> keys(n);
    if (threads <= 1 || n < 65536) {
        or_make_keys(&c, centers, cov, 0, n, keys.data());
        return or_counting_sort(keys.data(), n, order, sorted_keys);
    }
    // Parallel: keys by index chunks, then a per-chunk histogram, a
    // (bucket, chunk)-major prefix and a per-chunk scatter, which keeps the
    // result identical to the sequential stable sort.
    const uint32_t T = uint32_t(threads);
    const uint32_t chunk = (n + T - 1) / T;
    std::vector<std::vector<uint32_t>> hist(T, std::vector<uint32_t>(OR_BUCKETS, 0));
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < T; ++t)
        pool.emplace_back([&, t] {
            const uint32_t b = t * chunk, e = std::min(n, b + chunk);
            if (b >= e) return;
            or_make_keys(&c, centers, cov, b, e, keys.data());
            for (uint32_t i = b; i < e; ++i)
                if (keys[i] != OR_CULLED) ++hist[t][keys[i]];
        });
    for (auto& th : pool) th.join();
    pool.clear();
    uint32_t total = 0;
    for (uint32_t k = 0; k < OR_BUCKETS; ++k)
        for (uint32_t t = 0; t < T; ++t) {
            const uint32_t cnt = hist[t][k];
            hist[t][k] = total;
            total += cnt;
        }
    for (uint32_t t = 0; t < T; ++t)
        pool.emplace_back([&, t] {
            const uint32_t b = t * chunk, e = std::min(n, b + chunk);
            uint32_t* at = hist[t].data();
            for (uint32_t i = b; i < e; ++i) {
                const uint32_t k = keys[i];
                if (k == OR_CULLED) continue;
                const uint32_t dst = at[k]++;
                order[dst] = i;
                if (sorted_keys) sorted_keys[dst] = k;
            }
        });
    for (auto& th : pool) th.join();
    return total;
}

extern "C" uint32_t or_particle_key(const float* particle, const float eye[3], const float forward[3]) {
    const float age = particle[3], lifetime = particle[7];
    if (age >= lifetime) return OR_CULLED;                                   // particles.js:202
    const float dx = particle[0] - eye[0], dy = particle[1] - eye[1], dz = particle[2] - eye[2];
    const float dot = (dx * forward[0] + dy * forward[1]) + dz * forward[2];
    const float depth = std::fmax(dot, 1e-6f);                              // :203
    const float l = (float)log2l((long double)depth);
    const float v = ((l - -10.0f) * 4095.0f) / 30.0f;                        // :204
    const uint32_t bucket = (uint32_t)clampf(v, 0.0f, 4095.0f);
    return OR_PARTICLE_BUCKETS - 1u - bucket;                                // :205
}

extern "C" uint32_t or_particle_sort(const float* pool, uint32_t offset, uint32_t capacity, const float eye[3],
                                     const float forward[3], uint32_t* order, uint32_t* sorted_keys) {
    std::vector<uint32_t> keys(capacity);
    for (uint32_t i = 0; i < capacity; ++i) keys[i] = or_particle_key(pool + 8 * (size_t)(offset + i), eye, forward);
    const uint32_t live = or_counting_sort(keys.data(), capacity, order, sorted_keys);
    for (uint32_t j = 0; j < live; ++j) order[j] += offset;
    return live;
}

namespace {

// A half float's value (IEEE binary16), exactly.
float half_value(uint32_t h) {
    const uint32_t sign = (h >> 15) & 1u, e = (h >> 10) & 31u, m = h & 1023u;
    float v;
    if (e == 0)
        v = std::ldexp((float)m, -24);
    else if (e == 31)
        v = m ? NAN : INFINITY;
    else
        v = std::ldexp((float)(m | 1024u), (int)e - 25);
    return sign ? -v : v;
}

struct V3 {
    float r, g, b;
};
V3 coef(const uint32_t* sh, uint32_t words, uint32_t i, uint32_t k) {   // splats.js:338-344
    const size_t h = (size_t)i * words * 2 + k * 3;
    const uint32_t w0 = sh[h >> 1], w1 = sh[(h >> 1) + 1];
    const float a0 = half_value(w0 & 0xFFFFu), a1 = half_value(w0 >> 16);
    const float b0 = half_value(w1 & 0xFFFFu), b1 = half_value(w1 >> 16);
    return (h & 1) ? V3{a1, b0, b1} : V3{a0, a1, b0};
}
V3 mul(float s, V3 v) { return V3{s * v.r, s * v.g, s * v.b}; }
V3 add(V3 a, V3 b) { return V3{a.r + b.r, a.g + b.g, a.b + b.b}; }
V3 sub(V3 a, V3 b) { return V3{a.r - b.r, a.g - b.g, a.b - b.b}; }
uint32_t unorm8(float e) { return (uint32_t)std::floor(0.5f + 255.0f * clampf(e, 0.0f, 1.0f)); }

}  // namespace

extern "C" uint32_t or_shade(const float* centers, const uint32_t* sh, int degree, uint32_t i, const float eye[3]) {
    static const uint32_t coefficients[4] = {0, 3, 8, 15};
    const uint32_t words = (coefficients[degree] * 3 + 1) / 2;
    const float* c = centers + 4 * (size_t)i;
    const float vx = c[0] - eye[0], vy = c[1] - eye[1], vz = c[2] - eye[2];
    const float len = std::sqrt((vx * vx + vy * vy) + vz * vz);
    const float x = vx / len, y = vy / len, z = vz / len;
    V3 col = mul(0.4886025119029199f, sub(add(mul(-y, coef(sh, words, i, 0)), mul(z, coef(sh, words, i, 1))),
                                          mul(x, coef(sh, words, i, 2))));
    if (degree >= 2) {
        const float xx = x * x, yy = y * y, zz = z * z;
        V3 e = sub(mul(1.0925484305920792f * x * y, coef(sh, words, i, 3)),
                   mul(1.0925484305920792f * y * z, coef(sh, words, i, 4)));
        e = add(e, mul(0.31539156525252005f * (2.0f * zz - xx - yy), coef(sh, words, i, 5)));
        e = sub(e, mul(1.0925484305920792f * x * z, coef(sh, words, i, 6)));
        e = add(e, mul(0.5462742152960396f * (xx - yy), coef(sh, words, i, 7)));
        col = add(col, e);
        if (degree >= 3) {
            V3 h = add(mul(-0.5900435899266435f * y * (3.0f * xx - yy), coef(sh, words, i, 8)),
                       mul(2.890611442640554f * x * y * z, coef(sh, words, i, 9)));
            h = sub(h, mul(0.4570457994644658f * y * (4.0f * zz - xx - yy), coef(sh, words, i, 10)));
            h = add(h, mul(0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy), coef(sh, words, i, 11)));
            h = sub(h, mul(0.4570457994644658f * x * (4.0f * zz - xx - yy), coef(sh, words, i, 12)));
            h = add(h, mul(1.445305721320277f * z * (xx - yy), coef(sh, words, i, 13)));
            h = sub(h, mul(0.5900435899266435f * x * (xx - 3.0f * yy), coef(sh, words, i, 14)));
            col = add(col, h);
        }
    }
    uint32_t word;
    std::memcpy(&word, &c[3], 4);
    const float r = (float)(word & 255u) / 255.0f, g = (float)((word >> 8) & 255u) / 255.0f;
    const float b = (float)((word >> 16) & 255u) / 255.0f, a = (float)(word >> 24) / 255.0f;
    return unorm8(r + col.r) | (unorm8(g + col.g) << 8) | (unorm8(b + col.b) << 16) | (unorm8(a) << 24);
}

// ------------------------------------------------------------ capture readers

namespace {

// Double-double helpers (Knuth's two-sum, Dekker's split and product).
struct DD {
    double h, l;
};
DD dd_from_sum(double a, double b) {
    const double s = a + b, v = s - a;
    return {s, (a - (s - v)) + (b - v)};
}
DD dd_norm(double a, double b) {
    const double s = a + b;
    return {s, b - (s - a)};
}
DD dd_prod(double a, double b) {
    const double p = a * b;
    const double ca = 134217729.0 * a, ah = ca - (ca - a), al = a - ah;
    const double cb = 134217729.0 * b, bh = cb - (cb - b), bl = b - bh;
    return {p, (((ah * bh - p) + ah * bl) + al * bh) + al * bl};
}
DD operator+(DD a, DD b) {
    DD s = dd_from_sum(a.h, b.h);
    const DD t = dd_from_sum(a.l, b.l);
    s = dd_norm(s.h, s.l + t.h);
    return dd_norm(s.h, s.l + t.l);
}
DD operator*(DD a, DD b) {
    const DD p = dd_prod(a.h, b.h);
    return dd_norm(p.h, p.l + (a.h * b.l + a.l * b.h));
}
DD dd_over(DD a, double b) {
    const double q = a.h / b;
    const DD p = dd_prod(q, b);
    const DD r = dd_from_sum(a.h, -p.h);
    return dd_norm(q, ((r.h + (r.l - p.l)) + a.l) / b);
}

}  // namespace

// exp(x) = 2^k exp(r / 1024)^1024, r = x - k ln 2: a 13-term series for the
// small argument, ten squarings, all in double-double; then rounded once.
extern "C" double or_exp(double x) {
    if (std::isnan(x)) return x;
    if (x > 1000.0) return INFINITY;
    if (x < -1000.0) return 0.0;
    const double k = std::nearbyint(x / 0.6931471805599453);
    const DD ln2{6.93147180559945286227e-01, 2.31904681384629955842e-17};
    const DD kl = DD{k, 0.0} * ln2;
    const DD r = dd_over(DD{x, 0.0} + DD{-kl.h, -kl.l}, 1024.0);
    DD term{1.0, 0.0}, sum{1.0, 0.0};
    for (int n = 1; n <= 13; ++n) {
        term = dd_over(term * r, (double)n);
        sum = sum + term;
    }
    for (int s = 0; s < 10; ++s) sum = sum * sum;
    double y = sum.h;
    return std::ldexp(y, (int)k);
}

namespace {
double js_round(double x) {
    if (std::isnan(x) || std::isinf(x)) return x;
    const double f = std::floor(x);
    return (x - f >= 0.5) ? f + 1.0 : f;
}
uint32_t half_bits(double value) {   // render/hdr.js:152-163
    if (!(value > 0)) return 0;
    if (value >= 65504.0) return 0x7bff;
    if (value < std::ldexp(1.0, -24)) return 0;
    if (value < std::ldexp(1.0, -14)) return (uint32_t)js_round(value / std::ldexp(1.0, -24));
    int exponent = std::ilogb(value);
    uint32_t mantissa = (uint32_t)js_round((value / std::ldexp(1.0, exponent) - 1.0) * 1024.0);
    if (mantissa == 1024) {
        mantissa = 0;
        ++exponent;
    }
    return ((uint32_t)(exponent + 15) << 10) | mantissa;
}
}  // namespace

extern "C" uint32_t or_byte(double v) {
    const double r = std::fmax(0.0, std::fmin(255.0, js_round(v * 255.0)));
    return std::isnan(js_round(v * 255.0)) ? 0u : (uint32_t)r;
}

extern "C" uint32_t or_signed_half(double v) { return v < 0 ? (0x8000u | half_bits(-v)) : half_bits(v); }

namespace {

const uint32_t kCoefs[5] = {0, 3, 8, 15, 24};
const double kC0 = 0.28209479177387814;

// put() (scene/splats.js:335-369) with FP64 inputs; false for a bad position.
bool put_d(uint32_t i, double x, double y, double z, uint32_t colour, double sx, double sy, double sz, double qw,
           double qx, double qy, double qz, float* centers, float* cov, double bmin[3], double bmax[3]) {
    if (!(std::isfinite(x) && std::isfinite(y) && std::isfinite(z))) return false;
    float* c = centers + 4 * (size_t)i;
    c[0] = (float)x;
    c[1] = (float)y;
    c[2] = (float)z;
    std::memcpy(&c[3], &colour, 4);
    const double p[3] = {x + 0.0, y + 0.0, z + 0.0};
    for (int k = 0; k < 3; ++k) {
        if (p[k] < bmin[k]) bmin[k] = p[k];
        if (p[k] > bmax[k]) bmax[k] = p[k];
    }
    double length = v8_hypot4(qw, qx, qy, qz);
    if (!(length != 0.0)) length = 1.0;
    const double w = qw / length, u = qx / length, v = qy / length, t = qz / length;
    const double r00 = 1 - 2 * (v * v + t * t), r01 = 2 * (u * v - w * t), r02 = 2 * (u * t + w * v);
    const double r10 = 2 * (u * v + w * t), r11 = 1 - 2 * (u * u + t * t), r12 = 2 * (v * t - w * u);
    const double r20 = 2 * (u * t - w * v), r21 = 2 * (v * t + w * u), r22 = 1 - 2 * (u * u + v * v);
    const double m00 = r00 * sx, m01 = r01 * sy, m02 = r02 * sz;
    const double m10 = r10 * sx, m11 = r11 * sy, m12 = r12 * sz;
    const double m20 = r20 * sx, m21 = r21 * sy, m22 = r22 * sz;
    float* o = cov + 6 * (size_t)i;
    o[0] = (float)(m00 * m00 + m01 * m01 + m02 * m02);
    o[1] = (float)(m00 * m10 + m01 * m11 + m02 * m12);
    o[2] = (float)(m00 * m20 + m01 * m21 + m02 * m22);
    o[3] = (float)(m10 * m10 + m11 * m11 + m12 * m12);
    o[4] = (float)(m10 * m20 + m11 * m21 + m12 * m22);
    o[5] = (float)(m20 * m20 + m21 * m21 + m22 * m22);
    return true;
}

void put_sh(uint32_t* sh, uint32_t words, uint32_t i, uint32_t k, double r, double g, double b) {   // putSH
    uint16_t* halves = reinterpret_cast<uint16_t*>(sh);
    const size_t h = (size_t)i * words * 2 + k * 3;
    halves[h] = (uint16_t)or_signed_half(r);
    halves[h + 1] = (uint16_t)or_signed_half(g);
    halves[h + 2] = (uint16_t)or_signed_half(b);
}

double ply_value(const uint8_t* p, uint32_t type) {
    switch (type) {
        case 1: return (double)(int8_t)p[0];
        case 2: return (double)p[0];
        case 3: { int16_t v; std::memcpy(&v, p, 2); return v; }
        case 4: { uint16_t v; std::memcpy(&v, p, 2); return v; }
        case 5: { int32_t v; std::memcpy(&v, p, 4); return v; }
        case 6: { uint32_t v; std::memcpy(&v, p, 4); return v; }
        case 7: { float v; std::memcpy(&v, p, 4); return v; }
        case 8: { double v; std::memcpy(&v, p, 8); return v; }
        default: return 0.0;
    }
}

}  // namespace

extern "C" int or_decode_ply(const uint8_t* payload, uint32_t n, uint32_t stride, const uint32_t* types,
                             const uint32_t* offsets, uint32_t rest, float* centers, float* cov, uint32_t* sh,
                             double bmin[3], double bmax[3], uint32_t* bad) {
    for (int k = 0; k < 3; ++k) {
        bmin[k] = INFINITY;
        bmax[k] = -INFINITY;
    }
    const uint32_t per = rest / 3;
    const uint32_t words = (per * 3 + 1) / 2;
    for (uint32_t i = 0; i < n; ++i) {
        const uint8_t* rec = payload + (size_t)i * stride;
        auto f = [&](int k) { return ply_value(rec + offsets[k], types[k]); };
        const uint32_t colour = or_byte(0.5 + kC0 * f(3)) | (or_byte(0.5 + kC0 * f(4)) << 8) |
                                (or_byte(0.5 + kC0 * f(5)) << 16) |
                                (or_byte(1.0 / (1.0 + or_exp(-f(6)))) << 24);
        if (!put_d(i, f(0), f(1), f(2), colour, or_exp(f(7)), or_exp(f(8)), or_exp(f(9)), f(10), f(11), f(12),
                   f(13), centers, cov, bmin, bmax)) {
            *bad = i;
            return -4;
        }
        for (uint32_t k = 0; k < per; ++k) put_sh(sh, words, i, k, f(14 + k), f(14 + k + per), f(14 + k + 2 * per));
    }
    return 0;
}

extern "C" int or_decode_spz(const uint8_t* data, size_t len, uint32_t* count, uint32_t* degree, float* centers,
                             float* cov, uint32_t* sh, double bmin[3], double bmax[3], uint32_t* bad, char* err,
                             size_t errlen) {
    auto u32 = [&](size_t o) { uint32_t v; std::memcpy(&v, data + o, 4); return v; };
    if (len < 16 || u32(0) != 0x5053474eu) {
        std::snprintf(err, errlen, "splats: gzipped, but not a .spz");
        return -7;
    }
    const uint32_t version = u32(4);
    if (version < 1 || version > 3) {
        std::snprintf(err, errlen, "splats: a .spz of version %u; versions 1 to 3 are read", version);
        return -8;
    }
    const uint32_t n = u32(8), file_degree = data[12], fraction = data[13];
    if (file_degree > 4) {
        std::snprintf(err, errlen, "splats: a .spz with harmonics of degree %u", file_degree);
        return -9;
    }
    const uint32_t deg = std::min<uint32_t>(file_degree, 3), file_coefs = kCoefs[file_degree];
    const size_t pb = version == 1 ? 6 : 9, rb = version >= 3 ? 4 : 3;
    const size_t positions = 16, alphas = positions + n * pb, colours = alphas + n, scales = colours + n * 3;
    const size_t rotations = scales + n * 3, shs = rotations + n * rb, end = shs + (size_t)n * file_coefs * 3;
    if (n == 0) {
        std::snprintf(err, errlen, "splats: a .spz with no splats");
        return -10;
    }
    if (end > len) {
        std::snprintf(err, errlen, "splats: the .spz is cut short: %u splats need %zu bytes, it has %zu", n, end, len);
        return -11;
    }
    *count = n;
    *degree = deg;
    if (!centers) return 0;
    for (int k = 0; k < 3; ++k) {
        bmin[k] = INFINITY;
        bmax[k] = -INFINITY;
    }
    const double fixed = 1.0 / (double)(int32_t)(1u << (fraction & 31));
    const uint32_t words = (kCoefs[deg] * 3 + 1) / 2;
    static const double flip[15] = {-1, -1, 1, -1, 1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
    for (uint32_t i = 0; i < n; ++i) {
        double pos[3];
        for (int a = 0; a < 3; ++a) {
            if (version == 1) {
                uint16_t h;
                std::memcpy(&h, data + positions + i * 6 + a * 2, 2);
                const double sign = (h & 0x8000) ? -1.0 : 1.0;
                const int e = (h >> 10) & 31, m = h & 1023;
                pos[a] = e == 31 ? (m ? NAN : sign * INFINITY)
                                 : sign * (e == 0 ? m * std::ldexp(1.0, -24) : (1 + m / 1024.0) * std::ldexp(1.0, e - 15));
            } else {
                const uint8_t* p = data + positions + i * 9 + a * 3;
                int32_t v = (int32_t)(p[0] | (p[1] << 8) | (p[2] << 16));
                if (v & 0x800000) v -= 0x1000000;
                pos[a] = v * fixed;
            }
        }
        double q[4];
        if (rb == 3) {
            for (int a = 0; a < 3; ++a) q[a] = data[rotations + i * 3 + a] / 127.5 - 1;
            q[3] = std::sqrt(std::fmax(0.0, 1 - (q[0] * q[0] + q[1] * q[1] + q[2] * q[2])));
        } else {
            uint32_t packed = u32(rotations + i * 4);
            const uint32_t largest = packed >> 30;
            double sum = 0;
            for (int a = 3; a >= 0; --a) {
                if ((uint32_t)a == largest) continue;
                const uint32_t magnitude = packed & 511, negative = (packed >> 9) & 1;
                packed >>= 10;
                q[a] = 0.7071067811865476 * magnitude / 511 * (negative ? -1 : 1);
                sum += q[a] * q[a];
            }
            q[largest] = std::sqrt(std::fmax(0.0, 1 - sum));
        }
        uint32_t colour = (uint32_t)data[alphas + i] << 24;
        for (int k = 0; k < 3; ++k)
            colour |= or_byte(0.5 + kC0 * ((data[colours + i * 3 + k] / 255.0 - 0.5) / 0.15)) << (8 * k);
        double s3[3];
        for (int k = 0; k < 3; ++k) s3[k] = or_exp(data[scales + i * 3 + k] / 16.0 - 10);
        if (!put_d(i, pos[0], -pos[1], -pos[2], colour, s3[0], s3[1], s3[2], q[3], q[0], -q[1], -q[2], centers, cov,
                   bmin, bmax)) {
            *bad = i;
            return -4;
        }
        for (uint32_t k = 0; k < kCoefs[deg]; ++k) {
            const uint8_t* h = data + shs + (size_t)i * file_coefs * 3 + k * 3;
            put_sh(sh, words, i, k, (h[0] - 128) / 128.0 * flip[k], (h[1] - 128) / 128.0 * flip[k],
                   (h[2] - 128) / 128.0 * flip[k]);
        }
    }
    return 0;
}

// readSog's loop (scene/splats.js:167-199). Positions were stored as
// sign(x) ln(|x| + 1) in 16 bits over the means' range; rotations as the
// three smallest components of w x y z, the largest named by the alpha
// byte (252 + its index); colours, scales and harmonics through codebooks.
extern "C" int or_decode_sog(uint32_t n, uint32_t degree, const uint8_t* low, const uint8_t* high,
                             const uint8_t* quats, const uint8_t* scales, const uint8_t* sh0, const uint8_t* labels,
                             const uint8_t* palette, uint32_t palette_width, size_t palette_bytes,
                             const double mins[3], const double maxs[3], const double scale_book[256],
                             const double colour_book[256], const double sh_book[256], double sh_count,
                             float* centers, float* cov, uint32_t* sh, double bmin[3], double bmax[3], uint32_t* bad) {
    for (int k = 0; k < 3; ++k) {
        bmin[k] = INFINITY;
        bmax[k] = -INFINITY;
    }
    const uint32_t per = kCoefs[degree], words = (per * 3 + 1) / 2;
    for (uint32_t i = 0; i < n; ++i) {
        const size_t o = (size_t)i * 4;
        double m[3];
        for (int a = 0; a < 3; ++a) {
            const double v = (double)(low[o + a] | (high[o + a] << 8));
            double range = maxs[a] - mins[a];
            if (!(range != 0.0)) range = 1.0;   // (maxs - mins) || 1
            const double t = mins[a] + range * v / 65535.0;
            const double e = or_exp(std::fabs(t)) - 1.0;
            m[a] = t < 0 ? -e : e;
        }
        double q[4] = {1, 0, 0, 0};
        const uint32_t tag = quats[o + 3];
        if (tag >= 252) {
            const uint32_t largest = tag - 252;
            uint32_t k = 0;
            double sum = 0;
            for (uint32_t c = 0; c < 4; ++c) {
                if (c == largest) continue;
                q[c] = ((quats[o + k++] / 255.0) * 2.0 - 1.0) / 1.4142135623730951;
                sum += q[c] * q[c];
            }
            q[largest] = std::sqrt(std::fmax(0.0, 1.0 - sum));
        }
        uint32_t colour = (uint32_t)sh0[o + 3] << 24;
        for (int k = 0; k < 3; ++k) colour |= or_byte(0.5 + kC0 * colour_book[sh0[o + k]]) << (8 * k);
        const double sx = or_exp(scale_book[scales[o]]), sy = or_exp(scale_book[scales[o + 1]]),
                     sz = or_exp(scale_book[scales[o + 2]]);
        if (!put_d(i, m[0], m[1], m[2], colour, sx, sy, sz, q[0], q[1], q[2], q[3], centers, cov, bmin, bmax)) {
            *bad = i;
            return -4;
        }
        if (degree == 0) continue;
        const double label = (double)(labels[o] | (labels[o + 1] << 8));
        if (label >= sh_count) continue;
        const uint32_t lab = (uint32_t)label;
        const size_t row = (size_t)(lab / 64) * palette_width + (size_t)(lab % 64) * per;
        for (uint32_t k = 0; k < per; ++k) {
            const size_t c = (row + k) * 4;
            if (c + 2 >= palette_bytes) break;
            put_sh(sh, words, i, k, sh_book[palette[c]], sh_book[palette[c + 1]], sh_book[palette[c + 2]]);
        }
    }
    return 0;
}

// ------------------------------------------------------------------ draw

extern "C" void or_draw_tables(float srgb[256], float reach[256]) {
    for (int b = 0; b < 256; ++b) {
        const float c = (float)b / 255.0f;   // unpack4x8unorm
        if (c <= 0.04045f)
            srgb[b] = c / 12.92f;
        else
            srgb[b] = (float)powl((long double)((c + 0.055f) / 1.055f), 2.4L);
        reach[b] = (float)logl((long double)(255.0f * c));
    }
}

namespace {

// Cody and Waite's reduction, the Taylor polynomial to r^7 / 7!, 2^k.
float exp_pinned(float x) {
    if (std::isnan(x)) return x;
    if (x < -104.0f) return 0.0f;
    if (x > 88.0f) return INFINITY;
    const float k = rintf(x * 1.44269504f);
    const float r = (x - k * 0.693359375f) - k * -2.12194440e-4f;
    float p = 1.98412698e-4f;
    p = p * r + 1.38888889e-3f;
    p = p * r + 8.33333333e-3f;
    p = p * r + 4.16666667e-2f;
    p = p * r + 1.66666667e-1f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    int ki = (int)k;
    if (ki < -126) {
        p = p * std::ldexp(1.0f, ki + 126);
        ki = -126;
    }
    return p * std::ldexp(1.0f, ki);
}

}  // namespace

// A property check of the library's draw: its prepare step cuts each
// splat's pixel box to the pixels whose centre lies within the quad's
// half-extents (hx, hy) plus a margin of 1/64 pixel and 2^-16 of the extent.
// Over the splats of `order` this counts, out[0], the pixels in the pinned
// box that the coverage test covers and the cut leaves out (it must be 0),
// out[1] the covered pixels, out[2] the pinned box pixels and out[3] the cut
// box pixels.
extern "C" void or_draw_cut_check(const float* centers, const float* cov, const uint32_t* order, uint32_t count,
                                  const float mv[16], const float P[16], uint32_t width, uint32_t height,
                                  uint64_t out[4]) {
    float srgb[256], reach_t[256];
    or_draw_tables(srgb, reach_t);
    or_cloud c;
    std::memcpy(c.model_view, mv, sizeof(c.model_view));
    std::memcpy(c.projection, P, sizeof(c.projection));
    c.viewport[0] = (float)width;
    c.viewport[1] = (float)height;
    const float half_w = 0.5f * (float)width, half_h = 0.5f * (float)height;
    for (int k = 0; k < 4; ++k) out[k] = 0;
    for (uint32_t j = 0; j < count; ++j) {
        const uint32_t i = order[j];
        const float* p = centers + 4 * (size_t)i;
        float view[4], clip[4];
        for (int k = 0; k < 4; ++k)
            view[k] = ((mv[k] * p[0] + mv[4 + k] * p[1]) + mv[8 + k] * p[2]) + mv[12 + k] * 1.0f;
        for (int k = 0; k < 4; ++k)
            clip[k] = ((P[k] * view[0] + P[4 + k] * view[1]) + P[8 + k] * view[2]) + P[12 + k] * view[3];
        float f[3];
        or_footprint(&c, cov, i, view, f);
        const float a = f[0] + 0.3f, b = f[1], cc = f[2] + 0.3f;
        const float mid = 0.5f * (a + cc), hd = 0.5f * (a - cc);
        const float radius = std::sqrt(hd * hd + b * b);
        const float major = mid + radius, minor = mid - radius;
        uint32_t word;
        std::memcpy(&word, &p[3], 4);
        const float reach = reach_t[word >> 24];
        if (!(minor > 0.0f) || !(reach > 0.0f)) continue;
        float ax = 1.0f, ay = 0.0f;
        if (std::fabs(b) > 1e-12f) {
            const float ey = major - a;
            const float len = std::sqrt(b * b + ey * ey);
            ax = b / len;
            ay = ey / len;
        } else if (cc > a) {
            ax = 0.0f;
            ay = 1.0f;
        }
        const float la = std::fmin(std::sqrt(2.0f * major), 1024.0f);
        const float lc = std::fmin(std::sqrt(2.0f * minor), 1024.0f);
        const float ila = 1.0f / la, ilc = 1.0f / lc;
        const float qm = std::sqrt(std::fmin(reach, 4.0f));
        const float cx = (clip[0] / clip[3] + 1.0f) * half_w;
        const float cy = (1.0f - clip[1] / clip[3]) * half_h;
        const float hx = qm * (la * std::fabs(ax) + lc * std::fabs(ay));
        const float hy = qm * (la * std::fabs(ay) + lc * std::fabs(ax));
        if (!(std::isfinite(cx) && std::isfinite(cy) && std::isfinite(hx) && std::isfinite(hy))) continue;
        const float fx0 = std::fmax(std::floor((cx - hx) - 1.5f), 0.0f);
        const float fx1 = std::fmin(std::ceil((cx + hx) + 0.5f), (float)(width - 1));
        const float fy0 = std::fmax(std::floor((cy - hy) - 1.5f), 0.0f);
        const float fy1 = std::fmin(std::ceil((cy + hy) + 0.5f), (float)(height - 1));
        if (!(fx0 <= fx1 && fy0 <= fy1)) continue;
        // the cut, as the library's prepare step computes it
        const float mx = (hx + 0.015625f) + hx * (1.0f / 65536.0f);
        const float my = (hy + 0.015625f) + hy * (1.0f / 65536.0f);
        const float gx0 = std::fmax(fx0, std::ceil((cx - mx) - 0.5f));
        const float gx1 = std::fmin(fx1, std::floor((cx + mx) - 0.5f));
        const float gy0 = std::fmax(fy0, std::ceil((cy - my) - 0.5f));
        const float gy1 = std::fmin(fy1, std::floor((cy + my) - 0.5f));
        const bool cut_empty = !(gx0 <= gx1 && gy0 <= gy1);
        const int x0 = cut_empty ? 1 : (int)gx0, x1 = cut_empty ? 0 : (int)gx1;
        const int y0 = cut_empty ? 1 : (int)gy0, y1 = cut_empty ? 0 : (int)gy1;
        out[2] += (uint64_t)((int)fx1 - (int)fx0 + 1) * (uint64_t)((int)fy1 - (int)fy0 + 1);
        if (!cut_empty) out[3] += (uint64_t)(x1 - x0 + 1) * (uint64_t)(y1 - y0 + 1);
        for (int py = (int)fy0; py <= (int)fy1; ++py)
            for (int px = (int)fx0; px <= (int)fx1; ++px) {
                const float ex = ((float)px + 0.5f) - cx, ey = cy - ((float)py + 0.5f);
                const float ox = (ex * ax + ey * ay) * ila;
                const float oy = (ex * ay - ey * ax) * ilc;
                if (!(std::fabs(ox) <= qm && std::fabs(oy) <= qm)) continue;
                ++out[1];
                if (px < x0 || px > x1 || py < y0 || py > y1) ++out[0];
            }
    }
}

extern "C" void or_draw(const float* centers, const float* cov, const uint32_t* order, uint32_t count,
                        const uint32_t* shaded, const float mv[16], const float P[16], uint32_t width,
                        uint32_t height, float* image) {
    float srgb[256], reach_t[256];
    or_draw_tables(srgb, reach_t);
    or_cloud c;
    std::memcpy(c.model_view, mv, sizeof(c.model_view));
    std::memcpy(c.projection, P, sizeof(c.projection));
    c.viewport[0] = (float)width;
    c.viewport[1] = (float)height;
    const float half_w = 0.5f * (float)width, half_h = 0.5f * (float)height;
    for (uint32_t j = 0; j < count; ++j) {
        const uint32_t i = order[j];
        const float* p = centers + 4 * (size_t)i;
        float view[4], clip[4];
        for (int k = 0; k < 4; ++k)   // modelView * (x, y, z, 1), column sums
            view[k] = ((mv[k] * p[0] + mv[4 + k] * p[1]) + mv[8 + k] * p[2]) + mv[12 + k] * 1.0f;
        for (int k = 0; k < 4; ++k)
            clip[k] = ((P[k] * view[0] + P[4 + k] * view[1]) + P[8 + k] * view[2]) + P[12 + k] * view[3];
        float f[3];
        or_footprint(&c, cov, i, view, f);
        const float a = f[0] + 0.3f, b = f[1], cc = f[2] + 0.3f;
        const float mid = 0.5f * (a + cc), hd = 0.5f * (a - cc);
        const float radius = std::sqrt(hd * hd + b * b);
        const float major = mid + radius, minor = mid - radius;
        uint32_t word;
        if (shaded)
            word = shaded[i];
        else
            std::memcpy(&word, &p[3], 4);
        const float reach = reach_t[word >> 24];
        if (!(minor > 0.0f) || !(reach > 0.0f)) continue;
        float ax = 1.0f, ay = 0.0f;
        if (std::fabs(b) > 1e-12f) {
            const float ey = major - a;
            const float len = std::sqrt(b * b + ey * ey);
            ax = b / len;
            ay = ey / len;
        } else if (cc > a) {
            ax = 0.0f;
            ay = 1.0f;
        }
        const float la = std::fmin(std::sqrt(2.0f * major), 1024.0f);
        const float lc = std::fmin(std::sqrt(2.0f * minor), 1024.0f);
        const float ila = 1.0f / la, ilc = 1.0f / lc;
        const float qm = std::sqrt(std::fmin(reach, 4.0f));
        const float cx = (clip[0] / clip[3] + 1.0f) * half_w;
        const float cy = (1.0f - clip[1] / clip[3]) * half_h;
        const float hx = qm * (la * std::fabs(ax) + lc * std::fabs(ay));
        const float hy = qm * (la * std::fabs(ay) + lc * std::fabs(ax));
        if (!(std::isfinite(cx) && std::isfinite(cy) && std::isfinite(hx) && std::isfinite(hy))) continue;
        const float fx0 = std::fmax(std::floor((cx - hx) - 1.5f), 0.0f);
        const float fx1 = std::fmin(std::ceil((cx + hx) + 0.5f), (float)(width - 1));
        const float fy0 = std::fmax(std::floor((cy - hy) - 1.5f), 0.0f);
        const float fy1 = std::fmin(std::ceil((cy + hy) + 0.5f), (float)(height - 1));
        if (!(fx0 <= fx1 && fy0 <= fy1)) continue;
        const float alpha0 = (float)(word >> 24) / 255.0f;
        const float rgb[3] = {srgb[word & 255u], srgb[(word >> 8) & 255u], srgb[(word >> 16) & 255u]};
        for (int py = (int)fy0; py <= (int)fy1; ++py)
            for (int px = (int)fx0; px <= (int)fx1; ++px) {
                const float ex = ((float)px + 0.5f) - cx, ey = cy - ((float)py + 0.5f);
                const float ox = (ex * ax + ey * ay) * ila;
                const float oy = (ex * ay - ey * ax) * ilc;
                if (!(std::fabs(ox) <= qm && std::fabs(oy) <= qm)) continue;
                const float alpha = std::fmin(0.99f, exp_pinned(-(ox * ox + oy * oy)) * alpha0);
                if (alpha < 1.0f / 255.0f) continue;
                float* d = image + 4 * ((size_t)py * width + px);
                const float om = 1.0f - alpha;
                for (int k = 0; k < 3; ++k) d[k] = rgb[k] * alpha + d[k] * om;
                d[3] = alpha + d[3] * om;
            }
    }
}
