// all.cu -- single translation unit of the MOONS B200 library (the kernels
// live in headers shared by the entry-point files).
#include "mesh.cu"
#include "pcg.cu"
#include "mgpcg.cu"
#include "mhd.cu"
#include "noalloc.cu"
#include "unet.cu"
#include "diag.cu"
