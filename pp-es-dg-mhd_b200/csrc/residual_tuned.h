// residual_tuned.h -- written by autotune.py: residual tile per degree, fastest of the
// candidates timed on this GPU (residual ms per launch, vortex mesh of about 33 M DOFs).
//   p=1 (4, 8, 128, 4, 3): 0.3574 ms  <- chosen
//   p=1 (8, 4, 128, 4, 3): 0.3708 ms
//   p=1 (8, 8, 256, 2, 5): 0.3621 ms
//   p=1 (16, 4, 256, 2, 5): 0.3766 ms
#ifndef MHD_RES_CFG1
#define MHD_RES_CFG1 4, 8, 128, 4, 3
#endif
//   p=2 (8, 4, 256, 2, 5): 0.4457 ms  <- chosen
//   p=2 (4, 4, 128, 4, 3): 0.4605 ms
//   p=2 (8, 4, 256, 2, 4): 0.4496 ms
//   p=2 (4, 8, 256, 2, 5): 0.4509 ms
#ifndef MHD_RES_CFG2
#define MHD_RES_CFG2 8, 4, 256, 2, 5
#endif
//   p=3 (4, 4, 256, 2, 5): 0.6962 ms  <- chosen
//   p=3 (2, 4, 128, 4, 3): 0.7109 ms
//   p=3 (4, 4, 256, 2, 6): 0.6962 ms
//   p=3 (4, 2, 128, 4, 3): 0.7049 ms
#ifndef MHD_RES_CFG3
#define MHD_RES_CFG3 4, 4, 256, 2, 5
#endif
