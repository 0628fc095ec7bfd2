// Node N-API addon over libwsort.so: the JavaScript call that replaces
// SplatPass._encodeSort (src/render/splats.js:676-697) plus a readback.
//
// Not built here: Node and its headers are absent from this image and from
// the GPU machines (node-gyp would compile it with binding.gyp beside this
// file). The C ABI it binds is include/wsort.h; the Python binding
// (winding_b200/_lib.py) is the tested one.
//
//   const ws = require('./build/Release/wsort.node');
//   const ctx = ws.create(0);
//   const cloud = ws.loadSplats(ctx, bytes);            // Uint8Array: .splat / .ply / .spz
//   const {count, order, keys} = ws.sortSplats(ctx, cloud, {modelView, projection, viewport, cull});
//   ws.freeSplats(cloud);
//
// Errors are thrown as Error with the library's message (ws_last_error),
// which uses the reference's wording where it has one.
#include <node_api.h>

#include <cstdint>
#include <cstdio>
#include <cstring>

#include "wsort.h"

namespace {

struct Cloud {
    ws_ctx* ctx;
    ws_cloud* cloud;
};

bool check(napi_env env, napi_status s, const char* what) {
    if (s == napi_ok) return true;
    napi_throw_error(env, nullptr, what);
    return false;
}

napi_value undefined(napi_env env) {
    napi_value u;
    napi_get_undefined(env, &u);
    return u;
}

void throw_ws(napi_env env, ws_ctx* ctx, int rc, const char* fallback) {
    const char* msg = ctx ? ws_last_error(ctx) : nullptr;
    char code[16];
    std::snprintf(code, sizeof(code), "%d", rc);
    napi_throw_error(env, code, msg && *msg ? msg : fallback);
}

// Copies `n` numbers of obj[name] (a Float32Array, or an array of numbers)
// into out.
bool read_f32(napi_env env, napi_value obj, const char* name, float* out, size_t n) {
    napi_value v;
    if (!check(env, napi_get_named_property(env, obj, name, &v), "view: missing member")) return false;
    bool typed = false;
    napi_is_typedarray(env, v, &typed);
    if (typed) {
        napi_typedarray_type type;
        size_t length;
        void* data;
        napi_value ab;
        size_t offset;
        if (!check(env, napi_get_typedarray_info(env, v, &type, &length, &data, &ab, &offset), "view: bad array"))
            return false;
        if (type != napi_float32_array || length < n) {
            napi_throw_type_error(env, nullptr, "view: expected a Float32Array long enough");
            return false;
        }
        std::memcpy(out, data, n * sizeof(float));
        return true;
    }
    for (size_t k = 0; k < n; ++k) {
        napi_value e;
        double d;
        if (!check(env, napi_get_element(env, v, (uint32_t)k, &e), "view: bad array") ||
            !check(env, napi_get_value_double(env, e, &d), "view: expected numbers"))
            return false;
        out[k] = (float)d;
    }
    return true;
}

bool read_number(napi_env env, napi_value obj, const char* name, double* out) {
    napi_value v;
    return check(env, napi_get_named_property(env, obj, name, &v), "view: missing member") &&
           check(env, napi_get_value_double(env, v, out), "view: expected a number");
}

void finalize_ctx(napi_env, void* data, void*) { ws_destroy(static_cast<ws_ctx*>(data)); }

void finalize_cloud(napi_env, void* data, void*) {
    Cloud* c = static_cast<Cloud*>(data);
    if (c->cloud) ws_cloud_free(c->cloud);
    delete c;
}

// create(device) -> context
napi_value Create(napi_env env, napi_callback_info info) {
    size_t argc = 1;
    napi_value argv[1];
    napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
    int32_t device = 0;
    if (argc > 0) napi_get_value_int32(env, argv[0], &device);
    ws_ctx* ctx = nullptr;
    const int rc = ws_create(&ctx, device);
    if (rc) {
        throw_ws(env, nullptr, rc, "ws_create failed");
        return nullptr;
    }
    napi_value out;
    napi_create_external(env, ctx, finalize_ctx, nullptr, &out);
    return out;
}

// loadSplats(ctx, bytes) -> cloud (readSplats without a decoder,
// src/scene/splats.js:78-90)
napi_value LoadSplats(napi_env env, napi_callback_info info) {
    size_t argc = 2;
    napi_value argv[2];
    napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
    ws_ctx* ctx = nullptr;
    if (argc < 2 || !check(env, napi_get_value_external(env, argv[0], reinterpret_cast<void**>(&ctx)), "bad context"))
        return nullptr;
    napi_typedarray_type type;
    size_t length;
    void* data;
    napi_value ab;
    size_t offset;
    if (!check(env, napi_get_typedarray_info(env, argv[1], &type, &length, &data, &ab, &offset),
               "loadSplats: expected a Uint8Array"))
        return nullptr;
    ws_cloud* cloud = nullptr;
    const int rc = ws_cloud_load(ctx, static_cast<const uint8_t*>(data), length, &cloud);
    if (rc) {
        throw_ws(env, ctx, rc, "loadSplats failed");
        return nullptr;
    }
    Cloud* c = new Cloud{ctx, cloud};
    napi_value out;
    napi_create_external(env, c, finalize_cloud, nullptr, &out);
    return out;
}

// sortSplats(ctx, cloud, {modelView, projection, viewport, cull})
//   -> {count, order: Uint32Array, keys: Uint32Array}
napi_value SortSplats(napi_env env, napi_callback_info info) {
    size_t argc = 3;
    napi_value argv[3];
    napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
    ws_ctx* ctx = nullptr;
    Cloud* c = nullptr;
    if (argc < 3 || !check(env, napi_get_value_external(env, argv[0], reinterpret_cast<void**>(&ctx)), "bad context") ||
        !check(env, napi_get_value_external(env, argv[1], reinterpret_cast<void**>(&c)), "bad cloud"))
        return nullptr;
    ws_view v;
    double cull = 0.5;
    if (!read_f32(env, argv[2], "modelView", v.model_view, 16) || !read_f32(env, argv[2], "projection", v.projection, 16) ||
        !read_f32(env, argv[2], "viewport", v.viewport, 2) || !read_number(env, argv[2], "cull", &cull))
        return nullptr;
    v.cull = (float)cull;
    if (!c->cloud) {   // freed by freeSplats (src/render/splats.js:556)
        napi_throw_error(env, nullptr, "addSplats: these splats were unloaded; remove the node first");
        return nullptr;
    }
    uint32_t n = 0;
    int rc = ws_cloud_info(c->cloud, &n, nullptr, nullptr);
    if (rc) {
        throw_ws(env, ctx, rc, "ws_cloud_info failed");
        return nullptr;
    }
    void* order = nullptr;
    void* keys = nullptr;
    napi_value order_ab, keys_ab;
    if (!check(env, napi_create_arraybuffer(env, (size_t)(n ? n : 1) * 4, &order, &order_ab), "out of memory") ||
        !check(env, napi_create_arraybuffer(env, (size_t)(n ? n : 1) * 4, &keys, &keys_ab), "out of memory"))
        return nullptr;
    uint32_t count = 0;
    rc = ws_sort(ctx, c->cloud, &v, static_cast<uint32_t*>(order), static_cast<uint32_t*>(keys), &count,
                 WS_HOST_OUTPUT, nullptr);
    if (rc) {
        throw_ws(env, ctx, rc, "sortSplats failed");
        return nullptr;
    }
    napi_value result, count_v, order_v, keys_v;
    napi_create_object(env, &result);
    napi_create_uint32(env, count, &count_v);
    napi_create_typedarray(env, napi_uint32_array, count, order_ab, 0, &order_v);
    napi_create_typedarray(env, napi_uint32_array, count, keys_ab, 0, &keys_v);
    napi_set_named_property(env, result, "count", count_v);
    napi_set_named_property(env, result, "order", order_v);
    napi_set_named_property(env, result, "keys", keys_v);
    return result;
}

// freeSplats(cloud): Splats.destroy (src/render/splats.js:411-415); the
// handle is refused by every later call.
napi_value FreeSplats(napi_env env, napi_callback_info info) {
    size_t argc = 1;
    napi_value argv[1];
    napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
    Cloud* c = nullptr;
    if (argc < 1 || !check(env, napi_get_value_external(env, argv[0], reinterpret_cast<void**>(&c)), "bad cloud"))
        return nullptr;
    if (c->cloud) ws_cloud_free(c->cloud);
    c->cloud = nullptr;
    return undefined(env);
}

napi_value Init(napi_env env, napi_value exports) {
    const napi_property_descriptor props[] = {
        {"create", nullptr, Create, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"loadSplats", nullptr, LoadSplats, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"sortSplats", nullptr, SortSplats, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"freeSplats", nullptr, FreeSplats, nullptr, nullptr, nullptr, napi_default, nullptr},
    };
    napi_define_properties(env, exports, sizeof(props) / sizeof(props[0]), props);
    return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, Init)
