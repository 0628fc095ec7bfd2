/*
 * CPU oracle for the splat depth-key + stable counting-sort path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain C++ restatement of the
 * reference's arithmetic, used by the tests, by the smoke check and by the
 * CPU-baseline leg of the benchmark as the checker. The product library
 * (winding_b200/libwsort.so) never links, loads or calls it.
 *
 * What it restates (paths relative to the reference project):
 *   - the .splat record decode and covariance:   src/scene/splats.js:335-388
 *   - the per-cloud depth range (FP64):          src/render/splats.js:559-587
 *   - makeKeys and footprint (f32):              src/render/splats.js:102-124, :155-186
 *   - the stable order of survivors:             src/render/drawlist.js:186-229
 *   - an alpha emitter's particle keys:          src/render/particles.js:197-209
 *   - the shade pass (harmonics):                src/render/splats.js:333-381
 *   - the .ply and .spz readers' per-splat math: src/scene/splats.js:227-303, :398-468
 *   - the splat draw (vs / fs):                  src/render/splats.js:252-312
 *
 * Pinned evaluation order. WGSL lets a driver fuse and reorder f32 work, so
 * the oracle fixes one order and the CUDA kernels follow it bit for bit:
 * every f32 operation is a separately rounded IEEE op (built with
 * -ffp-contract=off, no fast-math), sums are taken left to right in the
 * order the WGSL source writes them, matrix-vector products are the
 * column sums col0*v0 + col1*v1 + col2*v2 + col3*v3, and divisions and
 * square roots are correctly rounded.
 */
#ifndef WSORT_ORACLE_H
#define WSORT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Number of 16-bit keys: render/splats.js:64 (BUCKETS). */
#define OR_BUCKETS 65536u
/* Marks a culled splat in the per-splat key array the oracle returns. */
#define OR_CULLED 0xFFFFFFFFu

/* The fields of the reference's Cloud uniform a sort depends on
 * (render/splats.js:80-92, filled at :574-587). */
typedef struct or_cloud {
    float model_view[16];
    float projection[16];
    float viewport[2];
    float depth_min;
    float depth_scale;
    uint32_t count;
    float cull;
} or_cloud;

/*
 * Decodes `nbytes` of .splat records (scene/splats.js:373-388, put :335-369).
 * centers: 4 f32 per splat (x, y, z, colour word bits); cov: 6 f32 per splat
 * (xx xy xz yy yz zz); bmin/bmax: the box around the centres, as doubles.
 * Returns 0, or -1 (length not a whole number of records, or zero),
 * -2 (a zip), -3 (gzip), -4 (non-finite position; *bad_index set),
 * -5 (a .ply header), -6 (a zstd .spz). The message text is left in err.
 */
int or_parse_splat(const uint8_t* bytes, size_t nbytes, float* centers, float* cov,
                   double bmin[3], double bmax[3], uint32_t* bad_index,
                   char* err, size_t errlen);

/*
 * The per-cloud depth range in FP64 (render/splats.js:561-582).
 * Returns 1 when the cloud is wholly behind the camera (far <= 0: the
 * reference skips it), else 0 with depth_min / depth_scale as the f32 values
 * the Cloud uniform holds.
 */
int or_depth_range(const float model_view[16], const double bmin[3], const double bmax[3],
                   float* depth_min, float* depth_scale);

/* Splat i's key (0..65535) or OR_CULLED: makeKeys (render/splats.js:155-186). */
uint32_t or_key(const or_cloud* c, const float* centers, const float* cov, uint32_t i);

/* footprint (render/splats.js:102-124): f[0]=xx, f[1]=xy, f[2]=yy. */
void or_footprint(const or_cloud* c, const float* cov, uint32_t i,
                  const float view[4], float f[3]);

/* Keys for splats [begin, end) into keys[i]. */
void or_make_keys(const or_cloud* c, const float* centers, const float* cov,
                  uint32_t begin, uint32_t end, uint32_t* keys);

/*
 * Stable counting sort of the survivors by (key, splat index): the order the
 * reference's DrawList.sort gives when survivors are pushed in index order.
 * Returns the survivor count S; order[0..S) and sorted_keys[0..S) are written.
 */
uint32_t or_counting_sort(const uint32_t* keys, uint32_t n, uint32_t* order,
                          uint32_t* sorted_keys);

/*
 * DrawList.sort restated as written (render/drawlist.js:186-229): LSD radix
 * over 4 bytes, skipping passes whose byte is constant. Sorts keys/payloads
 * in place (using the alt buffers as ping-pong space).
 */
void or_drawlist_sort(uint32_t* keys, uint32_t* payloads, uint32_t n,
                      uint32_t* keys_alt, uint32_t* payloads_alt);

/*
 * The whole per-view path: depth range, keys and the stable sort.
 * view_* are what a caller writes into the Cloud uniform; the range is
 * computed here. Returns S. threads > 1 splits the work across host threads
 * (deterministic: same output as threads == 1).
 */
uint32_t or_sort_view(const float* centers, const float* cov, uint32_t n,
                      const double bmin[3], const double bmax[3],
                      const float model_view[16], const float projection[16],
                      const float viewport[2], float cull,
                      uint32_t* order, uint32_t* sorted_keys, int threads);

/*
 * The shade pass for splat i (render/splats.js:371-381): its colour word as
 * seen from `eye` (the cloud's space), from its centre (4 f32, the 4th the
 * colour word's bits) and its harmonics of `degree` (1-3) in `sh`, packed as
 * scene/splats.js:306-333 packs them. Pinned order: normalize(v) is
 * v / sqrt((x x + y y) + z z); harmonics() (:347-368) is evaluated left to
 * right as written, each scalar chain (K x y) before it scales a
 * coefficient; unpack4x8unorm is byte / 255, pack4x8unorm
 * floor(0.5 + 255 clamp(e, 0, 1)), clamp giving the bound for NaN.
 */
uint32_t or_shade(const float* centers, const uint32_t* sh, int degree, uint32_t i, const float eye[3]);

/*
 * The capture readers' JavaScript arithmetic, pinned: Math.exp as the double
 * nearest the real value (the engines are within an ulp of it; a result
 * below 2^-1022 is rounded to a double, then to the subnormal grid), Math.round
 * with halves up, byte() = max(0, min(255, round(v 255))) with NaN as 0,
 * halfBits (render/hdr.js:152-163) and signedHalf (scene/splats.js:50-52).
 */
double or_exp(double x);
uint32_t or_byte(double v);
uint32_t or_signed_half(double v);

/*
 * parsePly's per-vertex loop (scene/splats.js:456-468) over `n` vertices of
 * `stride` bytes: fields[k] = (type, offset) of x y z f_dc_0..2 opacity
 * scale_0..2 rot_0..3 then f_rest_0.. (`rest` of them; types 1 int8, 2 uint8,
 * 3 int16, 4 uint16, 5 int32, 6 uint32, 7 float32, 8 float64). Writes 4 f32
 * a centre, 6 a covariance, and (rest > 0) shWords(degree) words a splat of
 * harmonics, degree the one with rest / 3 coefficients. Returns 0, or -4
 * with *bad the first vertex whose position is not finite. bmin / bmax: the
 * box, as the reader's doubles.
 */
int or_decode_ply(const uint8_t* payload, uint32_t n, uint32_t stride, const uint32_t* types,
                  const uint32_t* offsets, uint32_t rest, float* centers, float* cov, uint32_t* sh,
                  double bmin[3], double bmax[3], uint32_t* bad);

/*
 * parseSpz on gunzipped bytes (scene/splats.js:227-303): the header checks
 * (returns -7 not a .spz, -8 version, -9 degree, -10 no splats, -11 cut
 * short; message in err), then every splat. *count and *degree are set
 * first (call with centers NULL to learn them); sh gets shWords(degree)
 * words a splat. -4 with *bad as for .ply.
 */
int or_decode_spz(const uint8_t* data, size_t len, uint32_t* count, uint32_t* degree, float* centers, float* cov,
                  uint32_t* sh, double bmin[3], double bmax[3], uint32_t* bad, char* err, size_t errlen);

/*
 * readSog's per-splat loop (scene/splats.js:167-199) on images already
 * decoded and meta.json's numbers already read: pixel i of each image is its
 * bytes 4i .. 4i + 3 (labels and the palette only when degree > 0). mins,
 * maxs: the means' ranges; the codebooks hold 256 numbers each (NaN where
 * the reference's array has no entry); sh_count is shN.count as a number.
 * Returns 0, or -4 with *bad the first splat whose position is not finite.
 */
int or_decode_sog(uint32_t n, uint32_t degree, const uint8_t* low, const uint8_t* high, const uint8_t* quats,
                  const uint8_t* scales, const uint8_t* sh0, const uint8_t* labels, const uint8_t* palette,
                  uint32_t palette_width, size_t palette_bytes, const double mins[3], const double maxs[3],
                  const double scale_book[256], const double colour_book[256], const double sh_book[256],
                  double sh_count, float* centers, float* cov, uint32_t* sh, double bmin[3], double bmax[3],
                  uint32_t* bad);

/*
 * The splat draw (render/splats.js:252-312) as the library pins it: for each
 * of the first `count` splats of `order`, in order, the quad the vertex
 * shader builds and the fragments of the pixels whose centres its inverse
 * maps into [-e, e]^2, blended premultiplied over `image` (width x height
 * RGBA f32, row 0 at the top). shaded: colour words in place of the splats'
 * own, or NULL. srgb / reach: the 256-entry decodeSRGB and log tables this
 * oracle computes (or_draw_tables). See the library's draw for the pinned
 * rules; this restates them.
 */
void or_draw_tables(float srgb[256], float reach[256]);
/* The draw's box cut against the coverage test (the library's raster.cu,
 * prepare step): out = {covered pixels the cut leaves out, covered pixels,
 * pinned box pixels, cut box pixels}. */
void or_draw_cut_check(const float* centers, const float* cov, const uint32_t* order, uint32_t count,
                       const float mv[16], const float P[16], uint32_t width, uint32_t height, uint64_t out[4]);
void or_draw(const float* centers, const float* cov, const uint32_t* order, uint32_t count, const uint32_t* shaded,
             const float model_view[16], const float projection[16], uint32_t width, uint32_t height, float* image);

/* Depth buckets of an alpha emitter's sort: render/particles.js:44-48. */
#define OR_PARTICLE_BUCKETS 4096u

/*
 * Particle p's key (render/particles.js:197-205), or OR_CULLED for a dead
 * slot (age >= lifetime, :202). particle: its 8 f32 (position xyz, age,
 * velocity xyz, lifetime). depth = max(dot(position - eye, forward), 1e-6):
 * the dot product summed x, y, z in order; max returns the non-NaN operand.
 * bucket = u32(clamp(((log2(depth) - -10) * 4095) / 30, 0, 4095)), each f32
 * operation separately rounded and log2 the f32 nearest the real log2
 * (log2l rounded once to f32; WGSL leaves its accuracy open). Key
 * 4095 - bucket.
 */
uint32_t or_particle_key(const float* particle, const float eye[3], const float forward[3]);

/*
 * One emitter's sort: slots [offset, offset + capacity) of the pool (8 f32 a
 * particle), the live ones by (key, slot). order[] receives pool slot
 * indices; returns the live count.
 */
uint32_t or_particle_sort(const float* pool, uint32_t offset, uint32_t capacity, const float eye[3],
                          const float forward[3], uint32_t* order, uint32_t* sorted_keys);

#ifdef __cplusplus
}
#endif

#endif
