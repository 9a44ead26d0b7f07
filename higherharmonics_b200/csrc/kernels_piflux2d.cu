// Kernel instantiations for the PIFLUX2D model family.
#define HHG_MODEL hhg::PIFLUX2D
#define HHG_MODEL_NAME piflux2d
#include "hhg_launch.cuh"
