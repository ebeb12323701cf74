// residual2_tuned.h -- written by autotune.py: the fastest candidate per degree on this GPU
// (residual ms per launch, vortex mesh of about 33 M DOFs).
//   p=1 MHD_RES2_CFG (8, 8, 256, 2): 0.4201 ms
//   p=1 MHD_RES2_CFG (8, 4, 128, 4): 0.3827 ms  <- chosen
//   p=1 MHD_RES2_CFG (8, 6, 192, 3): 0.4248 ms
//   p=1 MHD_RES2_CFG (16, 4, 256, 2): 0.4260 ms
#ifndef MHD_RES2_CFG1
#define MHD_RES2_CFG1 8, 4, 128, 4
#endif
//   p=2 MHD_RES2_CFG (6, 4, 256, 2): 0.3765 ms
//   p=2 MHD_RES2_CFG (4, 3, 128, 4): 0.3573 ms  <- chosen
//   p=2 MHD_RES2_CFG (6, 3, 192, 3): 0.4291 ms
//   p=2 MHD_RES2_CFG (8, 3, 256, 2): 0.3679 ms
#ifndef MHD_RES2_CFG2
#define MHD_RES2_CFG2 4, 3, 128, 4
#endif
//   p=3 MHD_RES2_CFG (4, 4, 256, 2): 0.5768 ms
//   p=3 MHD_RES2_CFG (4, 2, 128, 4): 0.5697 ms  <- chosen
//   p=3 MHD_RES2_CFG (4, 3, 192, 3): 0.6483 ms
//   p=3 MHD_RES2_CFG (8, 2, 256, 2): 0.5903 ms
#ifndef MHD_RES2_CFG3
#define MHD_RES2_CFG3 4, 2, 128, 4
#endif
