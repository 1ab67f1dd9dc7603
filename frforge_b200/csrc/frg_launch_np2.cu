#include "frg_launch.cuh"
FRG_INSTANTIATE_NP(2)
