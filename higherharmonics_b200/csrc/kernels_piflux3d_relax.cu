// Kernel instantiations for the PIFLUX3D_RELAX model family.
#define HHG_MODEL hhg::PIFLUX3D_RELAX
#define HHG_MODEL_NAME piflux3d_relax
#include "hhg_launch.cuh"
