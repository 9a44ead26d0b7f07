// Kernel instantiations for the HONEYCOMB model family.
#define HHG_MODEL hhg::HONEYCOMB
#define HHG_MODEL_NAME honeycomb
#include "hhg_launch.cuh"
