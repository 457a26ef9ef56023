// Node N-API addon: Bearing's World calls the B200 solve stage through libbearing_gpu.so.
//
// Not built in this repository: node_api.h is not available here.  A maintainer builds it with
// node-gyp against include/bearing_gpu.h and links libbearing_gpu.so, with a binding.gyp whose
// one target lists this file, the include directory and the library's directory.  Every
// array handed over is one of World's or Contacts' own typed arrays (src/world.js:228-311,
// src/contact.js:184-248), passed by pointer with no copy.
#include <node_api.h>

#include <cstring>

#include "bearing_gpu.h"

namespace {

napi_value fail(napi_env env, const char* message) {
  napi_throw_error(env, nullptr, message);
  return nullptr;
}

// The data pointer of the typed array at obj[name], or nullptr (and a pending exception).
void* column(napi_env env, napi_value obj, const char* name, napi_typedarray_type want) {
  napi_value value;
  if (napi_get_named_property(env, obj, name, &value) != napi_ok) return nullptr;
  bool is = false;
  napi_is_typedarray(env, value, &is);
  if (!is) {
    napi_throw_type_error(env, nullptr, name);
    return nullptr;
  }
  napi_typedarray_type type;
  size_t length = 0, offset = 0;
  void* data = nullptr;
  napi_value buffer;
  napi_get_typedarray_info(env, value, &type, &length, &data, &buffer, &offset);
  if (type != want) {
    napi_throw_type_error(env, nullptr, name);
    return nullptr;
  }
  return data;
}

int32_t number(napi_env env, napi_value obj, const char* name) {
  napi_value value;
  int32_t out = 0;
  napi_get_named_property(env, obj, name, &value);
  napi_get_value_int32(env, value, &out);
  return out;
}

void finalize(napi_env, void* data, void*) { bg_destroy(static_cast<bg_ctx*>(data)); }

// create(device) -> an external holding a bg_ctx (World._setWorkers's place, src/world.js:516-524)
napi_value Create(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  int32_t device = 0;
  if (argc > 0) napi_get_value_int32(env, argv[0], &device);
  bg_ctx* ctx = bg_create(device, BG_FLAG_NONE);
  if (ctx == nullptr) return fail(env, "bearing-gpu: no usable CUDA device");
  napi_value out;
  napi_create_external(env, ctx, finalize, nullptr, &out);
  return out;
}

// World's and Contacts' own typed arrays as bg_bodies / bg_rows; false (with an exception
// pending) if one is missing or of the wrong type.  sliding, anchorA and anchorB stay NULL: after
// the stage only slipped() reads them, and the device runs it (src/contact.js:1122-1182).
void bodies(napi_env env, napi_value w, bg_bodies& B) {
  std::memset(&B, 0, sizeof B);
  B.capacity = number(env, w, "_capacity");
  B.awake_count = number(env, w, "_awakeCount");
  B.awake_list = static_cast<const int32_t*>(column(env, w, "_awakeList", napi_int32_array));
  B.awake = static_cast<const uint8_t*>(column(env, w, "_awake", napi_uint8_array));
  B.position = static_cast<double*>(column(env, w, "_position", napi_float64_array));
  B.rotation = static_cast<double*>(column(env, w, "_rotation", napi_float64_array));
  B.velocity = static_cast<double*>(column(env, w, "_velocity", napi_float64_array));
  B.angular = static_cast<double*>(column(env, w, "_angular", napi_float64_array));
  B.tumbled = static_cast<double*>(column(env, w, "_tumbled", napi_float64_array));
  B.ceiling = static_cast<double*>(column(env, w, "_ceiling", napi_float64_array));
  B.start = static_cast<double*>(column(env, w, "_start", napi_float64_array));
  B.start_q = static_cast<double*>(column(env, w, "_startQ", napi_float64_array));
  B.inv_i = static_cast<double*>(column(env, w, "_invI", napi_float64_array));
  B.inv_mass = static_cast<const double*>(column(env, w, "_invMass", napi_float64_array));
  B.inertia = static_cast<const double*>(column(env, w, "_inertia", napi_float64_array));
  B.inv_inertia = static_cast<const double*>(column(env, w, "_invInertia", napi_float64_array));
  B.dims = static_cast<const double*>(column(env, w, "_dims", napi_float64_array));
  B.damping = static_cast<const double*>(column(env, w, "_damping", napi_float64_array));
  B.angular_damping = static_cast<const double*>(column(env, w, "_angularDamping", napi_float64_array));
  B.gravity_scale = static_cast<const double*>(column(env, w, "_gravityScale", napi_float64_array));
  B.type = static_cast<const uint8_t*>(column(env, w, "_type", napi_uint8_array));
  B.shape = static_cast<const uint8_t*>(column(env, w, "_shape", napi_uint8_array));
  B.frozen = static_cast<const uint8_t*>(column(env, w, "_frozen", napi_uint8_array));
  B.framed = static_cast<const uint8_t*>(column(env, w, "_framed", napi_uint8_array));
  B.lock = static_cast<const uint8_t*>(column(env, w, "_lock", napi_uint8_array));
  B.joint_head = static_cast<const int32_t*>(column(env, w, "_jointHead", napi_int32_array));
}

bool views(napi_env env, napi_value w, napi_value c, bg_bodies& B, bg_rows& R) {
  bodies(env, w, B);
  std::memset(&R, 0, sizeof R);
  R.count = number(env, c, "count");
  R.solved = number(env, c, "solved");
  const int32_t* starts = static_cast<const int32_t*>(column(env, c, "starts", napi_int32_array));
  if (starts != nullptr) std::memcpy(R.starts, starts, sizeof R.starts);
  R.row = static_cast<const int32_t*>(column(env, c, "row", napi_int32_array));
  R.a = static_cast<const int32_t*>(column(env, c, "a", napi_int32_array));
  R.b = static_cast<const int32_t*>(column(env, c, "b", napi_int32_array));
  R.points = static_cast<const uint8_t*>(column(env, c, "points", napi_uint8_array));
  R.normal = static_cast<const double*>(column(env, c, "normal", napi_float64_array));
  R.t1 = static_cast<const double*>(column(env, c, "t1", napi_float64_array));
  R.t2 = static_cast<const double*>(column(env, c, "t2", napi_float64_array));
  R.friction = static_cast<const double*>(column(env, c, "friction", napi_float64_array));
  R.restitution = static_cast<const double*>(column(env, c, "restitution", napi_float64_array));
  R.tolerance = static_cast<const double*>(column(env, c, "tolerance", napi_float64_array));
  R.patch = static_cast<const double*>(column(env, c, "patch", napi_float64_array));
  R.separation = static_cast<const double*>(column(env, c, "separation", napi_float64_array));
  R.point = static_cast<const double*>(column(env, c, "point", napi_float64_array));
  R.shift = static_cast<const double*>(column(env, c, "shift", napi_float64_array));
  R.normal_impulse = static_cast<double*>(column(env, c, "normalImpulse", napi_float64_array));
  R.tangent_impulse1 = static_cast<double*>(column(env, c, "tangentImpulse1", napi_float64_array));
  R.tangent_impulse2 = static_cast<double*>(column(env, c, "tangentImpulse2", napi_float64_array));
  R.roll_impulse1 = static_cast<double*>(column(env, c, "rollImpulse1", napi_float64_array));
  R.roll_impulse2 = static_cast<double*>(column(env, c, "rollImpulse2", napi_float64_array));
  R.spin_impulse = static_cast<double*>(column(env, c, "spinImpulse", napi_float64_array));
  R.drift1 = static_cast<double*>(column(env, c, "drift1", napi_float64_array));
  R.drift2 = static_cast<double*>(column(env, c, "drift2", napi_float64_array));
  R.gap = static_cast<double*>(column(env, c, "gap", napi_float64_array));
  R.max_normal_impulse = static_cast<double*>(column(env, c, "maxNormalImpulse", napi_float64_array));
  R.relative_velocity = static_cast<double*>(column(env, c, "relativeVelocity", napi_float64_array));
  bool pending = false;
  napi_is_exception_pending(env, &pending);
  return !pending;
}

// solveStep(ctx, world, contacts, dt, substeps) -> 0 or a BG_E* code: src/world.js:962-1032.
napi_value SolveStep(napi_env env, napi_callback_info info) {
  size_t argc = 5;
  napi_value argv[5];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  if (argc < 5) return fail(env, "solveStep(ctx, world, contacts, dt, substeps)");
  bg_ctx* ctx = nullptr;
  napi_get_value_external(env, argv[0], reinterpret_cast<void**>(&ctx));
  napi_value w = argv[1], c = argv[2];
  bg_bodies B;
  bg_rows R;
  if (!views(env, w, c, B, R)) return nullptr;
  bg_step S;
  napi_get_value_double(env, argv[3], &S.dt);
  napi_get_value_int32(env, argv[4], &S.substeps);
  napi_value g;
  napi_get_named_property(env, w, "_gravity", &g);
  for (uint32_t k = 0; k < 3; k++) {
    napi_value x;
    napi_get_element(env, g, k, &x);
    napi_get_value_double(env, x, &S.gravity[k]);
  }
  napi_value out;
  napi_create_int32(env, bg_solve_step(ctx, &B, &R, &S), &out);
  return out;
}

// registerHost(ctx, world, contacts) -> 0 or a BG_E* code: page-locks the World's and Contacts'
// typed arrays in place (bg_register_host), for contacts.capacity rows.  Called once, and again
// whenever either has grown (Contacts._alloc, src/contact.js:184-255), so that solveStep copies
// them straight to and from the device.
napi_value RegisterHost(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  if (argc < 3) return fail(env, "registerHost(ctx, world, contacts)");
  bg_ctx* ctx = nullptr;
  napi_get_value_external(env, argv[0], reinterpret_cast<void**>(&ctx));
  bg_bodies B;
  bg_rows R;
  if (!views(env, argv[1], argv[2], B, R)) return nullptr;
  napi_value out;
  napi_create_int32(env, bg_register_host(ctx, &B, &R, number(env, argv[2], "capacity")), &out);
  return out;
}

void set_int(napi_env env, napi_value obj, const char* name, int32_t v) {
  napi_value x;
  napi_create_int32(env, v, &x);
  napi_set_named_property(env, obj, name, x);
}

// contactStep(ctx, world, list, dt, substeps, out) -> 0 or a BG_E* code: the step's whole contact
// side on the device (bg_contact_step).  list: {count, a, b, margin, tolerance, memory, reuse},
// the pairs narrow() reaches meet() with and each one's record; out: {points, touching} typed
// arrays of list.count, and on return rows, solved, pointsSolved and starts.
napi_value ContactStep(napi_env env, napi_callback_info info) {
  size_t argc = 6;
  napi_value argv[6];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  if (argc < 6) return fail(env, "contactStep(ctx, world, list, dt, substeps, out)");
  bg_ctx* ctx = nullptr;
  napi_get_value_external(env, argv[0], reinterpret_cast<void**>(&ctx));
  napi_value w = argv[1], l = argv[2], o = argv[5];
  bg_bodies B;
  bodies(env, w, B);
  bg_materials M;
  M.friction = static_cast<const double*>(column(env, w, "_friction", napi_float64_array));
  M.restitution = static_cast<const double*>(column(env, w, "_restitution", napi_float64_array));
  M.size = static_cast<const double*>(column(env, w, "_size", napi_float64_array));
  M.reach = static_cast<const double*>(column(env, w, "_reach", napi_float64_array));
  bg_contact_pairs P;
  P.list.count = number(env, l, "count");
  P.list.a = static_cast<const int32_t*>(column(env, l, "a", napi_int32_array));
  P.list.b = static_cast<const int32_t*>(column(env, l, "b", napi_int32_array));
  P.list.margin = static_cast<const double*>(column(env, l, "margin", napi_float64_array));
  P.list.tolerance = static_cast<const double*>(column(env, l, "tolerance", napi_float64_array));
  P.memory = static_cast<const int32_t*>(column(env, l, "memory", napi_int32_array));
  P.reuse = number(env, l, "reuse");
  bg_contact_result R;
  std::memset(&R, 0, sizeof R);
  R.points = static_cast<uint8_t*>(column(env, o, "points", napi_uint8_array));
  R.touching = static_cast<uint8_t*>(column(env, o, "touching", napi_uint8_array));
  bool pending = false;
  napi_is_exception_pending(env, &pending);
  if (pending) return nullptr;
  bg_step S;
  napi_get_value_double(env, argv[3], &S.dt);
  napi_get_value_int32(env, argv[4], &S.substeps);
  napi_value g;
  napi_get_named_property(env, w, "_gravity", &g);
  for (uint32_t k = 0; k < 3; k++) {
    napi_value x;
    napi_get_element(env, g, k, &x);
    napi_get_value_double(env, x, &S.gravity[k]);
  }
  const int32_t rc = bg_contact_step(ctx, &B, &M, &P, &S, &R);
  if (rc == BG_OK) {
    set_int(env, o, "rows", R.rows);
    set_int(env, o, "solved", R.solved);
    set_int(env, o, "pointsSolved", R.points_solved);
    napi_value starts;
    napi_create_array_with_length(env, BG_STARTS, &starts);
    for (uint32_t k = 0; k < BG_STARTS; k++) {
      napi_value x;
      napi_create_int32(env, R.starts[k], &x);
      napi_set_element(env, starts, k, x);
    }
    napi_set_named_property(env, o, "starts", starts);
  }
  napi_value out;
  napi_create_int32(env, rc, &out);
  return out;
}

napi_value LastError(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  bg_ctx* ctx = nullptr;
  napi_get_value_external(env, argv[0], reinterpret_cast<void**>(&ctx));
  napi_value out;
  napi_create_string_utf8(env, bg_last_error(ctx), NAPI_AUTO_LENGTH, &out);
  return out;
}

napi_value Init(napi_env env, napi_value exports) {
  napi_property_descriptor props[] = {
      {"create", nullptr, Create, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"solveStep", nullptr, SolveStep, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"registerHost", nullptr, RegisterHost, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"contactStep", nullptr, ContactStep, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"lastError", nullptr, LastError, nullptr, nullptr, nullptr, napi_default, nullptr},
  };
  napi_define_properties(env, exports, sizeof props / sizeof props[0], props);
  return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, Init)
