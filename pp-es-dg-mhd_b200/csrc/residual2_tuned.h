// residual2_tuned.h -- written by autotune.py: the fastest candidate per degree on this GPU
// (residual ms per launch, vortex mesh of about 33 M DOFs; set 0 stays unless another is faster by more
// than 1 %).
//   p=1 MHD_RES2_CFG (8, 4, 128, 4): 0.3356 ms  <- chosen
//   p=1 MHD_RES2_CFG (8, 4, 128, 5): 0.3388 ms
//   p=1 MHD_RES2_CFG (8, 4, 128, 6): 0.3582 ms
//   p=1 MHD_RES2_CFG (8, 8, 256, 3): 0.3502 ms
#ifndef MHD_RES2_CFG1
#define MHD_RES2_CFG1 8, 4, 128, 4
#endif
//   p=2 MHD_RES2_CFG (4, 3, 128, 4): 0.3422 ms  <- chosen
//   p=2 MHD_RES2_CFG (4, 3, 128, 5): 0.3485 ms
//   p=2 MHD_RES2_CFG (4, 3, 128, 6): 0.3884 ms
//   p=2 MHD_RES2_CFG (6, 4, 256, 3): 0.3824 ms
#ifndef MHD_RES2_CFG2
#define MHD_RES2_CFG2 4, 3, 128, 4
#endif
//   p=3 MHD_RES2_CFG (4, 2, 128, 4): 0.5782 ms  <- chosen
//   p=3 MHD_RES2_CFG (4, 2, 128, 5): 0.5750 ms
//   p=3 MHD_RES2_CFG (4, 2, 128, 6): 0.5965 ms
//   p=3 MHD_RES2_CFG (8, 2, 256, 3): 0.5918 ms
#ifndef MHD_RES2_CFG3
#define MHD_RES2_CFG3 4, 2, 128, 4
#endif
