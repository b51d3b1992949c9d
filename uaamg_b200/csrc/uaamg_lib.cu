// uaamg_lib.cu -- single translation unit of libuaamg_b200.so
#include "poisson.cu"
#include "batch.cu"
#include "mixed.cu"
#include "fp64ref.cu"
#include "viscosity.cu"
#include "projection.cu"
#include "extrapolate.cu"
#include "server.cu"
