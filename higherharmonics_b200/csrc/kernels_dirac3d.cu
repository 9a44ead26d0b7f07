// Kernel instantiations for the DIRAC3D model family.
#define HHG_MODEL hhg::DIRAC3D
#define HHG_MODEL_NAME dirac3d
#include "hhg_launch.cuh"
