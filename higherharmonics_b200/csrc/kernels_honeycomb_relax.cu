// Kernel instantiations for the HONEYCOMB_RELAX model family.
#define HHG_MODEL hhg::HONEYCOMB_RELAX
#define HHG_MODEL_NAME honeycomb_relax
#include "hhg_launch.cuh"
