// XLA custom-call (FFI) handler core: XLA's device buffers, in the operand orders that
// include/dmpc_xla.h lists, mapped onto dmpc_group / dmpc_adjoint and the C entry points.  The
// reference's JAX custom_vjp (diffmpc/solvers/sqp.py:572-801) is what a binding built on these
// replaces.  Every size is checked before any CUDA call.  The XLA handler symbols themselves are
// compiled only with -DDMPC_WITH_XLA_FFI and jaxlib's include directory (xla/ffi/api/ffi.h).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/dmpc.h"
#include "../../include/dmpc_xla.h"

namespace {

constexpr size_t kAlign = 256;  // dmpc_solve_fwd / dmpc_solve_adj workspace alignment

bool problem_ok(const dmpc_xla_problem* q, const dmpc_solver_params* p) {
  return q && p && q->batch >= 0 && q->nx >= 1 && q->nx <= DMPC_MAX_NX && q->nu >= 1 && q->nu <= DMPC_MAX_NU &&
         q->horizon >= 1 && q->n_model_params >= 0 && p->num_scp_iteration_max >= 1;
}

// Element counts of the shared problem-parameter operands 0-9 and of the trajectory shapes.
struct Shapes {
  uint64_t B, K, nx, nu, P, mi;
  uint64_t x() const { return B * nx; }
  uint64_t u() const { return B * nu; }
  uint64_t X() const { return B * K * nx; }
  uint64_t U() const { return B * K * nu; }
};

Shapes shapes_of(const dmpc_xla_problem* q, const dmpc_solver_params* p) {
  return Shapes{(uint64_t)q->batch, (uint64_t)q->horizon + 1, (uint64_t)q->nx, (uint64_t)q->nu,
                (uint64_t)q->n_model_params, (uint64_t)p->num_scp_iteration_max};
}

// A required buffer: exactly `elems` elements of `esize` bytes, non-null when non-empty.
bool exact(const dmpc_xla_buffer& b, uint64_t elems, uint64_t esize) {
  return b.bytes == elems * esize && (b.bytes == 0 || b.data != nullptr);
}
// An optional one: 0 bytes (absent) or exact.
bool optional(const dmpc_xla_buffer& b, uint64_t elems, uint64_t esize) { return b.bytes == 0 || exact(b, elems, esize); }
template <class T>
T* ptr(const dmpc_xla_buffer& b) {
  return b.bytes ? static_cast<T*>(b.data) : nullptr;
}

// Operands 0-9 (problem parameters, horizons) of both targets.
bool params_ok(const dmpc_xla_buffer* a, const Shapes& s) {
  return exact(a[0], s.B, 8) && exact(a[1], s.x(), 8) && exact(a[2], s.x(), 8) && exact(a[3], s.X(), 8) &&
         exact(a[4], s.U(), 8) && exact(a[5], s.x(), 8) && exact(a[6], s.u(), 8) && exact(a[7], s.x(), 8) &&
         exact(a[8], s.B * s.P, 8) && optional(a[9], s.B, 4);
}

void fill_group(dmpc_group& g, const dmpc_xla_problem* q, const dmpc_xla_buffer* a) {
  std::memset(&g, 0, sizeof(g));
  g.model = q->model;
  g.nx = q->nx;
  g.nu = q->nu;
  g.horizon = q->horizon;
  g.batch = q->batch;
  g.scheme = q->scheme;
  g.penalize_control_reference = q->penalize_control_reference;
  g.n_model_params = q->n_model_params;
  g.dt = ptr<const double>(a[0]);
  g.initial_state = ptr<const double>(a[1]);
  g.final_state = ptr<const double>(a[2]);
  g.reference_state = ptr<const double>(a[3]);
  g.reference_control = ptr<const double>(a[4]);
  g.w_x = ptr<const double>(a[5]);
  g.w_u = ptr<const double>(a[6]);
  g.w_f = ptr<const double>(a[7]);
  g.model_params = ptr<const double>(a[8]);
  g.horizons = ptr<const int32_t>(a[9]);
}

// The 256-byte aligned part of the workspace result, or nullptr if too small.
void* aligned_ws(const dmpc_xla_buffer& w, size_t need, size_t* bytes) {
  if (!w.data) return nullptr;
  const uintptr_t base = reinterpret_cast<uintptr_t>(w.data);
  const uintptr_t al = (base + kAlign - 1) / kAlign * kAlign;
  const size_t skip = (size_t)(al - base);
  if (w.bytes < skip || w.bytes - skip < need) return nullptr;
  *bytes = (size_t)(w.bytes - skip);
  return reinterpret_cast<void*>(al);
}

int copy_in(void* dst, const void* src, uint64_t bytes, cudaStream_t st) {
  if (bytes == 0 || dst == src) return DMPC_OK;
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st) == cudaSuccess ? DMPC_OK : DMPC_ERR_CUDA;
}

int zero(void* dst, uint64_t bytes, cudaStream_t st) {
  if (bytes == 0) return DMPC_OK;
  return cudaMemsetAsync(dst, 0, bytes, st) == cudaSuccess ? DMPC_OK : DMPC_ERR_CUDA;
}

}  // namespace

extern "C" const char* dmpc_xla_fwd_operands(void) {
  return "args: dt,initial_state,final_state,reference_state,reference_control,w_x,w_u,w_f,model_params,"
         "horizons,guess_states,guess_controls,guess_dual; "
         "rets: states,controls,dual,convergence_error,status,num_iter,convergence_errors,linesearch_alphas,"
         "num_pcg_iters,lin_states,lin_controls,workspace";
}

extern "C" const char* dmpc_xla_adj_operands(void) {
  return "args: dt,initial_state,final_state,reference_state,reference_control,w_x,w_u,w_f,model_params,"
         "horizons,states,controls,dual,lin_states,lin_controls,dl_dstates,dl_dcontrols,dual_backward_guess; "
         "rets: dual_backward,g_initial_state,g_final_state,g_w_x,g_w_u,g_w_f,g_reference_state,"
         "g_reference_control,g_model_params,num_pcg_iter,workspace";
}

extern "C" size_t dmpc_xla_workspace_size(const dmpc_xla_problem* q, const dmpc_solver_params* p) {
  if (!problem_ok(q, p)) return 0;
  dmpc_group g;
  dmpc_xla_buffer none[DMPC_XLA_FWD_ARGS] = {};
  fill_group(g, q, none);
  size_t n = dmpc_workspace_size(1, &g, p);
  // a ragged batch (horizons given) may take another CTA configuration: size for either
  static const int32_t kAnyHorizons = 0;
  g.horizons = &kAnyHorizons;  // only tested for presence on the host
  const size_t nr = dmpc_workspace_size(1, &g, p);
  if (n == 0 || nr == 0) return 0;
  return (nr > n ? nr : n) + kAlign;
}

extern "C" int dmpc_xla_solve_fwd(const dmpc_xla_problem* q, const dmpc_solver_params* p, const dmpc_xla_buffer* a,
                                  int n_args, const dmpc_xla_buffer* r, int n_rets, void* stream) {
  if (!problem_ok(q, p) || !a || !r || n_args != DMPC_XLA_FWD_ARGS || n_rets != DMPC_XLA_FWD_RETS)
    return DMPC_ERR_INVALID;
  const Shapes s = shapes_of(q, p);
  if (!params_ok(a, s) || !exact(a[10], s.X(), 8) || !exact(a[11], s.U(), 8) || !exact(a[12], s.X(), 8))
    return DMPC_ERR_INVALID;
  if (!exact(r[0], s.X(), 8) || !exact(r[1], s.U(), 8) || !exact(r[2], s.X(), 8) || !exact(r[3], s.B, 8) ||
      !exact(r[4], s.B, 4) || !exact(r[5], s.B, 4) || !exact(r[6], s.B * s.mi, 8) || !exact(r[7], s.B * s.mi, 8) ||
      !exact(r[8], s.B * s.mi, 4) || !exact(r[9], s.X(), 8) || !exact(r[10], s.U(), 8))
    return DMPC_ERR_INVALID;
  if (s.B == 0) return DMPC_OK;
  dmpc_group g;
  fill_group(g, q, a);
  g.states = ptr<double>(r[0]);
  g.controls = ptr<double>(r[1]);
  g.dual = ptr<double>(r[2]);
  g.convergence_error = ptr<double>(r[3]);
  g.status = ptr<int32_t>(r[4]);
  g.num_iter = ptr<int32_t>(r[5]);
  g.convergence_errors = ptr<double>(r[6]);
  g.linesearch_alphas = ptr<double>(r[7]);
  g.num_pcg_iters = ptr<int32_t>(r[8]);
  g.lin_states = ptr<double>(r[9]);
  g.lin_controls = ptr<double>(r[10]);
  const size_t need = dmpc_workspace_size(1, &g, p);
  if (need == 0) return DMPC_ERR_INVALID;
  size_t ws_bytes = 0;
  void* ws = aligned_ws(r[11], need, &ws_bytes);
  if (!ws) return DMPC_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = DMPC_OK;
  // the guess into the in/out arrays; histories and the guess's convergence error from zero
  if (rc == DMPC_OK) rc = copy_in(r[0].data, a[10].data, r[0].bytes, st);
  if (rc == DMPC_OK) rc = copy_in(r[1].data, a[11].data, r[1].bytes, st);
  if (rc == DMPC_OK) rc = copy_in(r[2].data, a[12].data, r[2].bytes, st);
  for (int k : {3, 6, 7, 8})
    if (rc == DMPC_OK) rc = zero(r[k].data, r[k].bytes, st);
  if (rc != DMPC_OK) return rc;
  return dmpc_solve_fwd(1, &g, p, ws, ws_bytes, stream);
}

extern "C" int dmpc_xla_solve_adj(const dmpc_xla_problem* q, const dmpc_solver_params* p,
                                  const int32_t* param_grad_index, int n_param_grads, const dmpc_xla_buffer* a,
                                  int n_args, const dmpc_xla_buffer* r, int n_rets, void* stream) {
  if (!problem_ok(q, p) || !a || !r || n_args != DMPC_XLA_ADJ_ARGS || n_rets != DMPC_XLA_ADJ_RETS)
    return DMPC_ERR_INVALID;
  if (n_param_grads < 0 || n_param_grads > DMPC_MAX_PARAM_GRADS || (n_param_grads > 0 && !param_grad_index))
    return DMPC_ERR_INVALID;
  const Shapes s = shapes_of(q, p);
  if (!params_ok(a, s) || !exact(a[10], s.X(), 8) || !exact(a[11], s.U(), 8) || !exact(a[12], s.X(), 8) ||
      !exact(a[13], s.X(), 8) || !exact(a[14], s.U(), 8) || !exact(a[15], s.X(), 8) || !exact(a[16], s.U(), 8) ||
      !optional(a[17], s.X(), 8))
    return DMPC_ERR_INVALID;
  if (!exact(r[0], s.X(), 8) || !optional(r[1], s.x(), 8) || !optional(r[2], s.x(), 8) || !optional(r[3], s.x(), 8) ||
      !optional(r[4], s.u(), 8) || !optional(r[5], s.x(), 8) || !optional(r[6], s.X(), 8) ||
      !optional(r[7], s.U(), 8) || !optional(r[8], s.B * (uint64_t)n_param_grads, 8) || !optional(r[9], s.B, 4))
    return DMPC_ERR_INVALID;
  if (n_param_grads > 0 && r[8].bytes == 0) return DMPC_ERR_INVALID;
  if (s.B == 0) return DMPC_OK;
  dmpc_group g;
  fill_group(g, q, a);
  // the forward solution; the adjoint reads the group's states, controls, dual and last
  // linearization point and writes none of them
  g.states = ptr<double>(a[10]);
  g.controls = ptr<double>(a[11]);
  g.dual = ptr<double>(a[12]);
  g.lin_states = ptr<double>(a[13]);
  g.lin_controls = ptr<double>(a[14]);
  dmpc_adjoint adj;
  std::memset(&adj, 0, sizeof(adj));
  adj.dl_dstates = ptr<const double>(a[15]);
  adj.dl_dcontrols = ptr<const double>(a[16]);
  adj.dual_backward_guess = ptr<const double>(a[17]);
  adj.dual_backward = ptr<double>(r[0]);
  adj.g_initial_state = ptr<double>(r[1]);
  adj.g_final_state = ptr<double>(r[2]);
  adj.g_w_x = ptr<double>(r[3]);
  adj.g_w_u = ptr<double>(r[4]);
  adj.g_w_f = ptr<double>(r[5]);
  adj.g_reference_state = ptr<double>(r[6]);
  adj.g_reference_control = ptr<double>(r[7]);
  adj.n_param_grads = n_param_grads;
  adj.param_grad_index = param_grad_index;
  adj.g_model_params = n_param_grads > 0 ? ptr<double>(r[8]) : nullptr;
  adj.num_pcg_iter = ptr<int32_t>(r[9]);
  const size_t need = dmpc_workspace_size(1, &g, p);
  if (need == 0) return DMPC_ERR_INVALID;
  size_t ws_bytes = 0;
  void* ws = aligned_ws(r[10], need, &ws_bytes);
  if (!ws) return DMPC_ERR_WORKSPACE;
  return dmpc_solve_adj(1, &g, &adj, p, ws, ws_bytes, stream);
}

// ------------------------------------------------------------------ XLA FFI handlers
// Built only against jaxlib's headers (-DDMPC_WITH_XLA_FFI -I<jaxlib>/include); jaxlib is not in
// the image this library is built in, so this part is unvalidated.  Operands are the variadic
// buffer lists of include/dmpc_xla.h; attributes: the problem's eight integers and the solver
// parameters as the raw bytes of a dmpc_solver_params (for the adjoint also the model-parameter
// indices whose gradients it computes).
#ifdef DMPC_WITH_XLA_FFI
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

template <class List>
bool gather(List& list, dmpc_xla_buffer* out, int n) {
  if ((int)list.size() != n) return false;
  for (int i = 0; i < n; ++i) {
    auto b = list.template get<ffi::AnyBuffer>(i);
    if (b.has_error()) return false;
    out[i] = dmpc_xla_buffer{b.value().untyped_data(), (uint64_t)b.value().size_bytes()};
  }
  return true;
}

template <class List>
bool gather_rets(List& list, dmpc_xla_buffer* out, int n) {
  if ((int)list.size() != n) return false;
  for (int i = 0; i < n; ++i) {
    auto b = list.template get<ffi::AnyBuffer>(i);
    if (b.has_error()) return false;
    out[i] = dmpc_xla_buffer{(*b.value())->untyped_data(), (uint64_t)(*b.value())->size_bytes()};
  }
  return true;
}

ffi::Error status(int rc) {
  return rc == DMPC_OK ? ffi::Error::Success()
                       : ffi::Error(rc == DMPC_ERR_INVALID ? ffi::ErrorCode::kInvalidArgument : ffi::ErrorCode::kInternal,
                                    dmpc_error_string(rc));
}

bool decode(int64_t model, int64_t nx, int64_t nu, int64_t horizon, int64_t batch, int64_t scheme, int64_t pcr,
            int64_t nmp, ffi::Span<const uint8_t> raw, dmpc_xla_problem* q, dmpc_solver_params* p) {
  if (raw.size() != sizeof(dmpc_solver_params)) return false;
  std::memcpy(p, raw.begin(), sizeof(*p));
  *q = dmpc_xla_problem{(int32_t)model, (int32_t)nx,     (int32_t)nu,  (int32_t)horizon,
                        (int32_t)batch, (int32_t)scheme, (int32_t)pcr, (int32_t)nmp};
  return true;
}

ffi::Error fwd_impl(cudaStream_t stream, ffi::RemainingArgs args, ffi::RemainingRets rets, int64_t model, int64_t nx,
                    int64_t nu, int64_t horizon, int64_t batch, int64_t scheme, int64_t pcr, int64_t nmp,
                    ffi::Span<const uint8_t> solver_params) {
  dmpc_xla_problem q;
  dmpc_solver_params p;
  dmpc_xla_buffer a[DMPC_XLA_FWD_ARGS], r[DMPC_XLA_FWD_RETS];
  if (!decode(model, nx, nu, horizon, batch, scheme, pcr, nmp, solver_params, &q, &p) ||
      !gather(args, a, DMPC_XLA_FWD_ARGS) || !gather_rets(rets, r, DMPC_XLA_FWD_RETS))
    return status(DMPC_ERR_INVALID);
  return status(dmpc_xla_solve_fwd(&q, &p, a, DMPC_XLA_FWD_ARGS, r, DMPC_XLA_FWD_RETS, stream));
}

ffi::Error adj_impl(cudaStream_t stream, ffi::RemainingArgs args, ffi::RemainingRets rets, int64_t model, int64_t nx,
                    int64_t nu, int64_t horizon, int64_t batch, int64_t scheme, int64_t pcr, int64_t nmp,
                    ffi::Span<const uint8_t> solver_params, ffi::Span<const int32_t> param_grad_index) {
  dmpc_xla_problem q;
  dmpc_solver_params p;
  dmpc_xla_buffer a[DMPC_XLA_ADJ_ARGS], r[DMPC_XLA_ADJ_RETS];
  if (!decode(model, nx, nu, horizon, batch, scheme, pcr, nmp, solver_params, &q, &p) ||
      !gather(args, a, DMPC_XLA_ADJ_ARGS) || !gather_rets(rets, r, DMPC_XLA_ADJ_RETS))
    return status(DMPC_ERR_INVALID);
  return status(dmpc_xla_solve_adj(&q, &p, param_grad_index.begin(), (int)param_grad_index.size(), a,
                                   DMPC_XLA_ADJ_ARGS, r, DMPC_XLA_ADJ_RETS, stream));
}

}  // namespace

#define DMPC_XLA_ATTRS                                                                                     \
  .Attr<int64_t>("model").Attr<int64_t>("nx").Attr<int64_t>("nu").Attr<int64_t>("horizon").Attr<int64_t>( \
      "batch").Attr<int64_t>("scheme").Attr<int64_t>("penalize_control_reference").Attr<int64_t>(        \
      "n_model_params").Attr<ffi::Span<const uint8_t>>("solver_params")

XLA_FFI_DEFINE_HANDLER_SYMBOL(dmpc_xla_fwd_handler, fwd_impl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .RemainingArgs()
                                  .RemainingRets() DMPC_XLA_ATTRS);
XLA_FFI_DEFINE_HANDLER_SYMBOL(dmpc_xla_adj_handler, adj_impl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .RemainingArgs()
                                  .RemainingRets() DMPC_XLA_ATTRS.Attr<ffi::Span<const int32_t>>("param_grad_index"));
#endif  // DMPC_WITH_XLA_FFI
