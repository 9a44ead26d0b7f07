// Kernel instantiations for the DIRAC2D model family.
#define HHG_MODEL hhg::DIRAC2D
#define HHG_MODEL_NAME dirac2d
#include "hhg_launch.cuh"
