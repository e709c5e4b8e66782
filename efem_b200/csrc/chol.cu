// Approximate-Jacobian Cholesky preconditioner (placeholder until the
// supernodal factorisation lands): reports the preconditioner as unavailable.
#include "efem_internal.h"

namespace efem {
struct Precond {};
efem_status precond_setup(Model&, int* ok, double* ms)
{
    *ok = 0;
    *ms = 0;
    set_error("the approximate-Jacobian preconditioner is not built in this version");
    return EFEM_ERR_UNSUPPORTED;
}
efem_status precond_apply(Model&, double*) { return EFEM_ERR_UNSUPPORTED; }
void free_precond(Model& m) { delete m.precond; m.precond = nullptr; }
void precond_info(const Model&, efem_model_info*) { }
}  // namespace efem
