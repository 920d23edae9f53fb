// Reference-element tables shared by the element kernels.
#pragma once

namespace cfem {
// Uploads the Tet10 reference tables (shape values, gradients, exact mass)
// to the constant memory of `device`. Idempotent per device.
int upload_tables(int device);
}  // namespace cfem
