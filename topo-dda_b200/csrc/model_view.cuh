// Read-only view of a model's device state for entry points that live in
// other translation units.
#pragma once

#include "operator.cuh"

namespace tdda {

struct ModelView {
    const ConvOperator<double2> *op;  // complex128 operator (tensor, plan)
    const double2 *al;                // 1/alpha per cell
    const long long *cell_of;         // dipole -> cell (device)
    const unsigned char *mask;        // cell in geometry, or nullptr for a full box
    long long N, nbox;
};

ModelView model_view(const tdda_model *m);

}  // namespace tdda
