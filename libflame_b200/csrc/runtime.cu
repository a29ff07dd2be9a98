// Library lifecycle, FLA_Obj objects, workspace and host<->device staging.
//
// Replaces src/base/flamec/main/FLA_Init.c, FLA_Obj.c, FLA_Check.c of the
// reference: same entry points and semantics, with object buffers in HBM.
#include <climits>
#include <cstring>
#include <mutex>

#include "common.h"

namespace fb {

static Context g_ctx;
Context& ctx() { return g_ctx; }

static std::string g_last_error;
static unsigned int g_error_level = FLA_FULL_ERROR_CHECKING;
static unsigned long g_next_id = 1;

void set_last_error(const std::string& msg) {
  g_last_error = msg;
  std::fprintf(stderr, "libflame_b200: %s\n", msg.c_str());
}

void check_fail(const char* func, const char* what) {
  // Same behaviour as FLA_Check_error_code(): message, then abort().
  std::fprintf(stderr, "libflame: %s: %s\n", func, what);
  std::fflush(stderr);
  std::abort();
}

// ---------------------------------------------------------------------------
// Workspace slots.
// ---------------------------------------------------------------------------
struct WsBuf {
  void* p = nullptr;
  size_t bytes = 0;
};
static WsBuf g_ws[WS_NSLOTS];

void* ws_get(int slot, size_t bytes) {
  WsBuf& w = g_ws[slot];
  if (bytes == 0) bytes = 256;
  if (w.bytes >= bytes) return w.p;
  if (w.p) {
    cudaStreamSynchronize(ctx().stream);
    cudaStreamSynchronize(ctx().side);
    cudaFree(w.p);
    w.p = nullptr;
    w.bytes = 0;
  }
  size_t want = bytes + bytes / 8;  // a little slack to limit regrowth
  if (cudaMalloc(&w.p, want) != cudaSuccess) {
    cudaGetLastError();
    if (cudaMalloc(&w.p, bytes) != cudaSuccess) {
      cudaGetLastError();
      set_last_error("workspace allocation failed");
      w.p = nullptr;
      return nullptr;
    }
    want = bytes;
  }
  w.bytes = want;
  return w.p;
}

void ws_release_all() {
  for (auto& w : g_ws) {
    if (w.p) cudaFree(w.p);
    w.p = nullptr;
    w.bytes = 0;
  }
}

bool is_device_ptr(const void* ptr) {
  cudaPointerAttributes at;
  cudaError_t e = cudaPointerGetAttributes(&at, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// ---------------------------------------------------------------------------
// Device timing.
// ---------------------------------------------------------------------------
static cudaEvent_t g_op_ev[2] = {nullptr, nullptr};
static bool g_op_open = false;
static float g_last_op_ms = 0.0f;
static bool g_prof = false;
struct ProfRec {
  cudaEvent_t a = nullptr, b = nullptr;
  int cls = 0;
  double flops = 0.0;
};
static std::vector<ProfRec> g_prof_recs;
static size_t g_prof_used = 0;
static double g_prof_ms[PROF_NCLASS], g_prof_flops[PROF_NCLASS];
static unsigned long long g_prof_n[PROF_NCLASS];

// While an enclosing driver holds the op window (op_hold), the op_begin /
// op_end / collection of the drivers it calls are no-ops, so the window
// spans the whole enclosing call.
static bool g_op_hold = false;
void op_hold(bool on) { g_op_hold = on; }

// The library's streams are non-blocking, so they are not ordered after
// work the caller left on the default stream (a tensor library producing the
// input, a pending copy).  Every call first makes its main stream wait for
// an event recorded on the legacy default stream, which completes after all
// work previously issued to it and to every blocking stream: the call then
// sees the caller's data as a synchronous CPU library would.  (A caller
// producing the input on its own non-blocking stream synchronizes first.)
void order_after_caller() {
  static cudaEvent_t ev = nullptr;
  if (!ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  cudaEventRecord(ev, cudaStreamLegacy);
  cudaStreamWaitEvent(ctx().stream, ev, 0);
}

void op_begin(cudaStream_t st) {
  if (g_op_hold) return;
  order_after_caller();
  if (!g_op_ev[0]) {
    cudaEventCreate(&g_op_ev[0]);
    cudaEventCreate(&g_op_ev[1]);
  }
  cudaEventRecord(g_op_ev[0], st);
  g_op_open = true;
}

void op_end(cudaStream_t st) {
  if (!g_op_open || g_op_hold) return;
  cudaEventRecord(g_op_ev[1], st);
}

static void prof_collect() {
  if (g_op_open && !g_op_hold) {
    cudaEventSynchronize(g_op_ev[1]);
    cudaEventElapsedTime(&g_last_op_ms, g_op_ev[0], g_op_ev[1]);
    g_op_open = false;
  }
  for (size_t i = 0; i < g_prof_used; ++i) {
    ProfRec& r = g_prof_recs[i];
    float ms = 0.0f;
    cudaEventSynchronize(r.b);
    cudaEventElapsedTime(&ms, r.a, r.b);
    g_prof_ms[r.cls] += ms;
    g_prof_flops[r.cls] += r.flops;
    g_prof_n[r.cls] += 1;
  }
  g_prof_used = 0;
}

bool prof_on() { return g_prof; }

int prof_begin(cudaStream_t st) {
  if (!g_prof) return -1;
  if (g_prof_used == g_prof_recs.size()) {
    ProfRec r;
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    g_prof_recs.push_back(r);
  }
  int slot = (int)g_prof_used++;
  cudaEventRecord(g_prof_recs[slot].a, st);
  return slot;
}

void prof_end(int slot, cudaStream_t st, int cls, double flops) {
  if (slot < 0) return;
  ProfRec& r = g_prof_recs[slot];
  r.cls = cls;
  r.flops = flops;
  cudaEventRecord(r.b, st);
}

int sync_all() {
  FB_CK(cudaStreamSynchronize(ctx().side));
  FB_CK(cudaStreamSynchronize(ctx().stream));
  prof_collect();
  return FLA_SUCCESS;
}

int status_reset() {
  Context& c = ctx();
  op_begin(c.stream);
  FB_CK(cudaMemsetAsync(c.d_status, 0, sizeof(int) * ST_WORDS, c.stream));
  // info slot: INT_MAX means "no failure"; kernels atomicMin into it.
  int big = INT_MAX;
  FB_CK(cudaMemcpyAsync(c.d_status + ST_INFO, &big, sizeof(int), cudaMemcpyHostToDevice, c.stream));
  return FLA_SUCCESS;
}

int status_read(int* info) {
  Context& c = ctx();
  op_end(c.stream);
  FB_CK(cudaMemcpyAsync(c.h_status, c.d_status, sizeof(int) * 2, cudaMemcpyDeviceToHost, c.stream));
  FB_CK(cudaStreamSynchronize(c.stream));
  prof_collect();
  if (c.h_status[ST_ERROR] != 0) {
    set_last_error("a kernel wait exceeded its iteration limit (error flag " +
                   std::to_string(c.h_status[ST_ERROR]) + ")");
    return FLA_FAILURE;
  }
  if (info) *info = (c.h_status[ST_INFO] == INT_MAX) ? -1 : c.h_status[ST_INFO];
  return FLA_SUCCESS;
}

// ---------------------------------------------------------------------------
// Staging of FLA_Obj views.
// ---------------------------------------------------------------------------
static size_t dt_size(FLA_Datatype dt) {
  switch (dt) {
    case FLA_FLOAT: return 4;
    case FLA_DOUBLE: return 8;
    case FLA_INT: return 4;
    case FLA_COMPLEX: return 8;
    case FLA_DOUBLE_COMPLEX: return 16;
    default: return 8;
  }
}

int stage(const FLA_Obj& A, int slot, Staged* s, bool copy_in, bool need_align) {
  Context& c = ctx();
  order_after_caller();
  s->m = (long)A.m;
  s->n = (long)A.n;
  s->esize = dt_size(A.base->datatype);
  char* buf = (char*)A.base->buffer;
  long rs = (long)A.base->rs, cs = (long)A.base->cs;
  s->orig = buf + ((long)A.offm * rs + (long)A.offn * cs) * (long)s->esize;
  s->orig_ld = cs;
  s->orig_is_host = !is_device_ptr(A.base->buffer);
  bool aligned = ((reinterpret_cast<uintptr_t>(s->orig) & 15u) == 0) &&
                 ((cs * (long)s->esize) % 16 == 0);
  if (!s->orig_is_host && (aligned || !need_align)) {
    s->dev = s->orig;
    s->ld = cs;
    s->staged = false;
    return FLA_SUCCESS;
  }
  // Copy into workspace with a padded leading dimension (multiple of 16 B).
  long ld = s->m > 0 ? s->m : 1;
  long mult = 16 / (long)s->esize;
  if (mult < 1) mult = 1;
  ld = ((ld + mult - 1) / mult) * mult;
  size_t bytes = (size_t)ld * (size_t)(s->n > 0 ? s->n : 1) * s->esize;
  void* d = ws_get(slot, bytes);
  if (!d) return FLA_FAILURE;
  s->dev = d;
  s->ld = ld;
  s->staged = true;
  if (copy_in && s->m > 0 && s->n > 0) {
    FB_CK(cudaMemcpy2DAsync(d, (size_t)ld * s->esize, s->orig, (size_t)cs * s->esize,
                            (size_t)s->m * s->esize, (size_t)s->n, cudaMemcpyDefault, c.stream));
  }
  return FLA_SUCCESS;
}

int unstage(const Staged& s, bool copy_out) {
  Context& c = ctx();
  if (!s.staged || !copy_out || s.m == 0 || s.n == 0) return FLA_SUCCESS;
  FB_CK(cudaMemcpy2DAsync(s.orig, (size_t)s.orig_ld * s.esize, s.dev, (size_t)s.ld * s.esize,
                          (size_t)s.m * s.esize, (size_t)s.n, cudaMemcpyDefault, c.stream));
  return FLA_SUCCESS;
}

}  // namespace fb

using namespace fb;

// ===========================================================================
// C ABI: lifecycle.
// ===========================================================================
extern "C" {

void FLA_Init(void) {
  Context& c = ctx();
  if (c.initialized) return;
  if (cudaGetDevice(&c.device) != cudaSuccess) {
    cudaGetLastError();
    c.device = 0;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, c.device) != cudaSuccess) {
    set_last_error("FLA_Init: no CUDA device available");
    std::abort();
  }
  c.num_sms = prop.multiProcessorCount;
  c.smem_optin = prop.sharedMemPerBlockOptin;
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  cudaStreamCreateWithPriority(&c.stream, cudaStreamNonBlocking, lo);
  cudaStreamCreateWithPriority(&c.side, cudaStreamNonBlocking, hi);
  for (auto& e : c.ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  cudaMalloc(&c.d_status, sizeof(int) * ST_WORDS);
  cudaMallocHost(&c.h_status, sizeof(int) * ST_WORDS);
  cudaMemset(c.d_status, 0, sizeof(int) * ST_WORDS);
  c.launches = 0;
  c.initialized = true;
}

void FLA_Finalize(void) {
  Context& c = ctx();
  if (!c.initialized) return;
  cudaDeviceSynchronize();
  ws_release_all();
  for (auto& e : c.ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  if (c.stream) cudaStreamDestroy(c.stream);
  if (c.side) cudaStreamDestroy(c.side);
  if (c.d_status) cudaFree(c.d_status);
  if (c.h_status) cudaFreeHost(c.h_status);
  c.stream = c.side = nullptr;
  c.d_status = nullptr;
  c.h_status = nullptr;
  c.initialized = false;
}

FLA_Bool FLA_Initialized(void) { return ctx().initialized ? TRUE : FALSE; }

// src/base/flamec/main/FLA_Init.c:95-127: initialise only if needed and
// remember whether this call did it.
void FLA_Init_safe(FLA_Error* init_result) {
  if (FLA_Initialized()) {
    *init_result = FLA_FAILURE;
  } else {
    FLA_Init();
    *init_result = FLA_SUCCESS;
  }
}

void FLA_Finalize_safe(FLA_Error init_result) {
  if (init_result == FLA_SUCCESS) FLA_Finalize();
}

unsigned int FLA_Check_error_level(void) { return g_error_level; }

unsigned int FLA_Check_error_level_set(unsigned int level) {
  unsigned int old = g_error_level;
  g_error_level = level;
  return old;
}

unsigned long long FLA_B200_kernel_launches(void) { return ctx().launches; }

double FLA_B200_last_op_ms(void) { return (double)g_last_op_ms; }

void FLA_B200_profile(int on) {
  g_prof = on != 0;
  for (int i = 0; i < PROF_NCLASS; ++i) {
    g_prof_ms[i] = 0.0;
    g_prof_flops[i] = 0.0;
    g_prof_n[i] = 0;
  }
  g_prof_used = 0;
}

int FLA_B200_profile_read(int cls, double* ms, double* flops, unsigned long long* launches) {
  if (cls < 0 || cls >= PROF_NCLASS) return FLA_FAILURE;
  if (ms) *ms = g_prof_ms[cls];
  if (flops) *flops = g_prof_flops[cls];
  if (launches) *launches = g_prof_n[cls];
  return FLA_SUCCESS;
}
const char* FLA_B200_last_error(void) { return g_last_error.c_str(); }
int FLA_B200_num_sms(void) { return ctx().num_sms; }

// ===========================================================================
// C ABI: objects (src/base/flamec/main/FLA_Obj.c).
// ===========================================================================
static void obj_init_base(FLA_Base_obj* b, FLA_Datatype dt, dim_t m, dim_t n) {
  std::memset(b, 0, sizeof(*b));
  b->datatype = dt;
  b->elemtype = FLA_SCALAR;  // flat (FLA_Obj.c:57); FLA_MATRIX marks hierarchical objects
  b->m = m;
  b->n = n;
  b->m_inner = m;
  b->n_inner = n;
  b->id = g_next_id++;
  b->uplo = FLA_FULL_MATRIX;
}

static void obj_init_view(FLA_Obj* obj, FLA_Base_obj* b, dim_t m, dim_t n) {
  obj->offm = 0;
  obj->offn = 0;
  obj->m = m;
  obj->n = n;
  obj->m_inner = m;
  obj->n_inner = n;
  obj->base = b;
}

FLA_Error FLA_Obj_create_without_buffer(FLA_Datatype datatype, dim_t m, dim_t n, FLA_Obj* obj) {
  FB_REQUIRE(obj != nullptr, "FLA_Obj_create_without_buffer", "null object pointer");
  FB_REQUIRE(datatype >= FLA_FLOAT && datatype <= FLA_CONSTANT, "FLA_Obj_create_without_buffer",
             "invalid datatype");
  FLA_Base_obj* b = (FLA_Base_obj*)std::malloc(sizeof(FLA_Base_obj));
  obj_init_base(b, datatype, m, n);
  obj_init_view(obj, b, m, n);
  return FLA_SUCCESS;
}

FLA_Error FLA_Obj_create(FLA_Datatype datatype, dim_t m, dim_t n, dim_t rs, dim_t cs,
                         FLA_Obj* obj) {
  FB_REQUIRE(obj != nullptr, "FLA_Obj_create", "null object pointer");
  if (!ctx().initialized) FLA_Init();
  FLA_Obj_create_without_buffer(datatype, m, n, obj);
  // FLA_Obj.c:55-70: rs = cs = 0 selects column-major storage.
  if (rs == 0 && cs == 0) {
    rs = 1;
    cs = m > 0 ? m : 1;
  }
  FB_REQUIRE(rs == 1, "FLA_Obj_create", "only column-major objects (rs == 1) are supported");
  FB_REQUIRE(cs >= m, "FLA_Obj_create", "column stride smaller than the number of rows");
  size_t es = dt_size(datatype);
  size_t elems = (size_t)cs * (size_t)(n > 0 ? n : 1);
  void* p = nullptr;
  if (cudaMalloc(&p, elems * es) != cudaSuccess) {
    cudaGetLastError();
    set_last_error("FLA_Obj_create: cudaMalloc failed");
    return FLA_FAILURE;
  }
  cudaMemset(p, 0, elems * es);
  FLA_Base_obj* b = obj->base;
  b->rs = rs;
  b->cs = cs;
  b->buffer = p;
  b->n_elem_alloc = elems;
  b->b200_owns_device_buffer = 1;
  return FLA_SUCCESS;
}

FLA_Error FLA_Obj_attach_buffer(void* buffer, dim_t rs, dim_t cs, FLA_Obj* obj) {
  FB_REQUIRE(obj != nullptr && obj->base != nullptr, "FLA_Obj_attach_buffer", "null object");
  // FLA_Obj.c:522-537 (with FLA_Obj_attach_buffer_check): rs = cs = 0 means
  // column-major with ld = m.
  if (rs == 0 && cs == 0) {
    rs = 1;
    cs = obj->base->m > 0 ? obj->base->m : 1;
  }
  FB_REQUIRE(buffer != nullptr || obj->base->m == 0 || obj->base->n == 0, "FLA_Obj_attach_buffer",
             "null buffer");
  FLA_Base_obj* b = obj->base;
  b->buffer = buffer;
  b->rs = rs;
  b->cs = cs;
  b->b200_owns_device_buffer = 0;
  return FLA_SUCCESS;
}

FLA_Error FLA_Obj_free(FLA_Obj* obj) {
  if (obj == nullptr || obj->base == nullptr) return FLA_SUCCESS;
  FLA_Base_obj* b = obj->base;
  if (b->b200_owns_device_buffer && b->buffer) {
    cudaDeviceSynchronize();
    cudaFree(b->buffer);
  }
  std::free(b);
  obj->base = nullptr;
  obj->m = obj->n = 0;
  return FLA_SUCCESS;
}

FLA_Error FLA_Obj_free_without_buffer(FLA_Obj* obj) {
  if (obj == nullptr || obj->base == nullptr) return FLA_SUCCESS;
  std::free(obj->base);
  obj->base = nullptr;
  obj->m = obj->n = 0;
  return FLA_SUCCESS;
}

FLA_Datatype FLA_Obj_datatype(FLA_Obj obj) { return obj.base ? obj.base->datatype : FLA_CONSTANT; }
dim_t FLA_Obj_length(FLA_Obj obj) { return obj.m; }
dim_t FLA_Obj_width(FLA_Obj obj) { return obj.n; }
dim_t FLA_Obj_min_dim(FLA_Obj obj) { return obj.m < obj.n ? obj.m : obj.n; }
dim_t FLA_Obj_max_dim(FLA_Obj obj) { return obj.m > obj.n ? obj.m : obj.n; }
dim_t FLA_Obj_row_stride(FLA_Obj obj) { return obj.base ? obj.base->rs : 0; }
dim_t FLA_Obj_col_stride(FLA_Obj obj) { return obj.base ? obj.base->cs : 0; }

void* FLA_Obj_buffer_at_view(FLA_Obj obj) {
  if (!obj.base || !obj.base->buffer) return nullptr;
  char* b = (char*)obj.base->buffer;
  return b + (obj.offm * obj.base->rs + obj.offn * obj.base->cs) * dt_size(obj.base->datatype);
}

}  // extern "C"
