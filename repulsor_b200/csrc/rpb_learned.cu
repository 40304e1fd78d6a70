// Learned per-cluster preconditioner (filled in by the MLP implementation).
#include <string>

#include "rpb_internal.cuh"
#include "rpb_mesh.cuh"

namespace rpb {

rpb_status learned_precondition(rpb_mesh* m, double, double, const double*, double*)
{
    (void)m;
    set_error("the learned preconditioner has not been trained for this mesh");
    return RPB_EINVAL;
}

}  // namespace rpb
