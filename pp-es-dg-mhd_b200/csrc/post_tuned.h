// post_tuned.h -- written by autotune.py: the fastest candidate per degree on this GPU
// (ms per SSP-RK3 step (OEDG + LDF + PP), vortex mesh of about 33 M DOFs).
//   p=1 MHD_PP_CFG (256, 4); MHD_SIG_CFG (8, 8, 3): 1.7010 ms  <- chosen
//   p=1 MHD_PP_CFG (128, 8); MHD_SIG_CFG (8, 4, 4): 1.7123 ms
//   p=1 MHD_PP_CFG (256, 3); MHD_SIG_CFG (16, 4, 3): 1.7176 ms
//   p=1 MHD_PP_CFG (192, 5); MHD_SIG_CFG (4, 8, 4): 1.7356 ms
#ifndef MHD_PP_CFG1
#define MHD_PP_CFG1 256, 4
#endif
#ifndef MHD_SIG_CFG1
#define MHD_SIG_CFG1 8, 8, 3
#endif
//   p=2 MHD_PP_CFG (256, 4); MHD_SIG_CFG (8, 4, 3): 1.8810 ms  <- chosen
//   p=2 MHD_PP_CFG (128, 8); MHD_SIG_CFG (4, 4, 4): 1.9303 ms
//   p=2 MHD_PP_CFG (256, 3); MHD_SIG_CFG (8, 2, 3): 1.9478 ms
//   p=2 MHD_PP_CFG (512, 2); MHD_SIG_CFG (4, 8, 3): 1.9111 ms
#ifndef MHD_PP_CFG2
#define MHD_PP_CFG2 256, 4
#endif
#ifndef MHD_SIG_CFG2
#define MHD_SIG_CFG2 8, 4, 3
#endif
//   p=3 MHD_PP_CFG (256, 4); MHD_SIG_CFG (4, 4, 2): 2.7732 ms  <- chosen
//   p=3 MHD_PP_CFG (128, 8); MHD_SIG_CFG (4, 2, 3): 2.8388 ms
//   p=3 MHD_PP_CFG (256, 3); MHD_SIG_CFG (4, 3, 2): 2.8616 ms
//   p=3 MHD_PP_CFG (192, 5); MHD_SIG_CFG (2, 4, 3): 2.8784 ms
#ifndef MHD_PP_CFG3
#define MHD_PP_CFG3 256, 4
#endif
#ifndef MHD_SIG_CFG3
#define MHD_SIG_CFG3 4, 4, 2
#endif
