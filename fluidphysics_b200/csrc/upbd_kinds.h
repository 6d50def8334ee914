// Kernel classes of the per-kernel timing (upbd_profile_frame,
// upbd_batch_profile_frame); names through upbd_kernel_name.
#pragma once

namespace upbd {

enum KernelKind {
  K_INTEGRATE, K_SCAN, K_SCATTER, K_RANKFIX, K_DENSITY, K_DISP, K_APPLY_FLUID, K_COLLECT,
  K_SOLID_SOLVE, K_APPLY_SOLID, K_SOLVE_TETS, K_SOLID_CONTACTS, K_APPLY_SOLID_CONTACTS,
  K_BOND_CONTACTS, K_APPLY_BOUNDS_VEL, K_SOLID_VISC, K_XSPH, K_XSPH_APPLY, K_EMIT, K_CUT,
  K_COUNT_ACTIVE, K_NUM_KINDS
};

extern const char* const kKernelNames[K_NUM_KINDS];

}  // namespace upbd
