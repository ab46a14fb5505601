/* Declarations of the Node-API functions the addon (home-measure-privacy_b200/node/gsb200_addon.cc)
 * uses, with the signatures of the public Node-API documentation (N-API version 8), so that a
 * CPU test can compile-check the addon where Node.js is not installed.  node-gyp builds the
 * addon against Node's own node_api.h; this file is only for that check. */
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct napi_env__* napi_env;
typedef struct napi_value__* napi_value;
typedef struct napi_ref__* napi_ref;
typedef struct napi_callback_info__* napi_callback_info;
typedef struct napi_deferred__* napi_deferred;
typedef struct napi_async_work__* napi_async_work;
typedef enum { napi_ok, napi_invalid_arg, napi_object_expected, napi_string_expected, napi_name_expected, napi_function_expected, napi_number_expected, napi_boolean_expected, napi_array_expected, napi_generic_failure, napi_pending_exception, napi_cancelled } napi_status;
typedef enum { napi_undefined, napi_null, napi_boolean, napi_number, napi_string, napi_symbol, napi_object, napi_function, napi_external, napi_bigint } napi_valuetype;
typedef enum { napi_int8_array, napi_uint8_array, napi_uint8_clamped_array, napi_int16_array, napi_uint16_array, napi_int32_array, napi_uint32_array, napi_float32_array, napi_float64_array, napi_bigint64_array, napi_biguint64_array } napi_typedarray_type;
typedef napi_value (*napi_callback)(napi_env env, napi_callback_info info);
typedef void (*napi_finalize)(napi_env env, void* finalize_data, void* finalize_hint);
typedef void (*napi_async_execute_callback)(napi_env env, void* data);
typedef void (*napi_async_complete_callback)(napi_env env, napi_status status, void* data);
#define NAPI_AUTO_LENGTH SIZE_MAX
napi_status napi_create_string_utf8(napi_env, const char*, size_t, napi_value*);
napi_status napi_create_error(napi_env, napi_value code, napi_value msg, napi_value* result);
napi_status napi_create_int32(napi_env, int32_t, napi_value*);
napi_status napi_create_double(napi_env, double, napi_value*);
napi_status napi_set_named_property(napi_env, napi_value, const char*, napi_value);
napi_status napi_get_named_property(napi_env, napi_value, const char*, napi_value*);
napi_status napi_has_named_property(napi_env, napi_value, const char*, bool*);
napi_status napi_throw(napi_env, napi_value);
napi_status napi_throw_error(napi_env, const char* code, const char* msg);
napi_status napi_throw_type_error(napi_env, const char* code, const char* msg);
napi_status napi_get_cb_info(napi_env, napi_callback_info, size_t* argc, napi_value* argv, napi_value* this_arg, void** data);
napi_status napi_get_value_external(napi_env, napi_value, void**);
napi_status napi_create_external(napi_env, void*, napi_finalize, void*, napi_value*);
napi_status napi_is_typedarray(napi_env, napi_value, bool*);
napi_status napi_is_array(napi_env, napi_value, bool*);
napi_status napi_get_typedarray_info(napi_env, napi_value, napi_typedarray_type*, size_t*, void**, napi_value*, size_t*);
napi_status napi_typeof(napi_env, napi_value, napi_valuetype*);
napi_status napi_get_value_double(napi_env, napi_value, double*);
napi_status napi_get_value_int32(napi_env, napi_value, int32_t*);
napi_status napi_get_value_int64(napi_env, napi_value, int64_t*);
napi_status napi_get_value_bool(napi_env, napi_value, bool*);
napi_status napi_get_element(napi_env, napi_value, uint32_t, napi_value*);
napi_status napi_get_array_length(napi_env, napi_value, uint32_t*);
napi_status napi_create_arraybuffer(napi_env, size_t, void**, napi_value*);
napi_status napi_create_typedarray(napi_env, napi_typedarray_type, size_t, napi_value, size_t, napi_value*);
napi_status napi_create_reference(napi_env, napi_value, uint32_t, napi_ref*);
napi_status napi_delete_reference(napi_env, napi_ref);
napi_status napi_get_reference_value(napi_env, napi_ref, napi_value*);
napi_status napi_create_promise(napi_env, napi_deferred*, napi_value*);
napi_status napi_resolve_deferred(napi_env, napi_deferred, napi_value);
napi_status napi_reject_deferred(napi_env, napi_deferred, napi_value);
napi_status napi_create_async_work(napi_env, napi_value, napi_value, napi_async_execute_callback, napi_async_complete_callback, void*, napi_async_work*);
napi_status napi_queue_async_work(napi_env, napi_async_work);
napi_status napi_delete_async_work(napi_env, napi_async_work);
napi_status napi_get_undefined(napi_env, napi_value*);
napi_status napi_create_object(napi_env, napi_value*);
napi_status napi_create_function(napi_env, const char*, size_t, napi_callback, void*, napi_value*);
#ifdef __cplusplus
}
#endif
#define NAPI_MODULE(name, fn) extern "C" napi_value napi_register_module_v1(napi_env env, napi_value exports) { return fn(env, exports); }
#define NODE_GYP_MODULE_NAME gsb200
