// residual_tuned.h -- written by autotune.py: residual tile per degree, fastest of the
// candidates timed on this GPU (residual ms per launch, vortex mesh of about 33 M DOFs).
//   p=1 (8, 4, 128, 4, 3): 0.3869 ms  <- chosen
//   p=1 (8, 4, 128, 4, 2): 0.4224 ms
//   p=1 (8, 8, 256, 2, 6): 0.3876 ms
//   p=1 (16, 4, 256, 2, 5): 0.3968 ms
#ifndef MHD_RES_CFG1
#define MHD_RES_CFG1 8, 4, 128, 4, 3
#endif
//   p=2 (4, 4, 128, 4, 2): 0.4767 ms
//   p=2 (4, 4, 128, 4, 3): 0.4657 ms
//   p=2 (8, 4, 256, 2, 5): 0.4570 ms  <- chosen
//   p=2 (4, 2, 128, 4, 2): 0.6776 ms
#ifndef MHD_RES_CFG2
#define MHD_RES_CFG2 8, 4, 256, 2, 5
#endif
//   p=3 (4, 2, 128, 4, 3): 0.7662 ms
//   p=3 (4, 2, 128, 4, 2): 0.8550 ms
//   p=3 (4, 4, 256, 2, 5): 0.7665 ms
//   p=3 (2, 4, 128, 4, 3): 0.7608 ms  <- chosen
#ifndef MHD_RES_CFG3
#define MHD_RES_CFG3 2, 4, 128, 4, 3
#endif
