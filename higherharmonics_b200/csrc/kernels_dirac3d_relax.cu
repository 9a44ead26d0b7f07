// Kernel instantiations for the DIRAC3D_RELAX model family.
#define HHG_MODEL hhg::DIRAC3D_RELAX
#define HHG_MODEL_NAME dirac3d_relax
#include "hhg_launch.cuh"
