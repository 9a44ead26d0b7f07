// Kernel instantiations for the PIFLUX2D_SYM model family.
#define HHG_MODEL hhg::PIFLUX2D_SYM
#define HHG_MODEL_NAME piflux2d_sym
#include "hhg_launch.cuh"
