// Launchers of the ETD2RK passes for a 1024^2 grid (FP64 and FP32).
#include "chns_launch.cuh"
CHNS_INSTANTIATE(1024)
