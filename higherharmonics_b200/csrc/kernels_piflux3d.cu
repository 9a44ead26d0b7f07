// Kernel instantiations for the PIFLUX3D model family.
#define HHG_MODEL hhg::PIFLUX3D
#define HHG_MODEL_NAME piflux3d
#include "hhg_launch.cuh"
