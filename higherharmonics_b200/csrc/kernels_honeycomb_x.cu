// Kernel instantiations for the HONEYCOMB_X model family.
#define HHG_MODEL hhg::HONEYCOMB_X
#define HHG_MODEL_NAME honeycomb_x
#include "hhg_launch.cuh"
