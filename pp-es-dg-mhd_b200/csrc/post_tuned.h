// post_tuned.h -- written by autotune.py: the fastest candidate per degree on this GPU
// (ms per SSP-RK3 step (OEDG + LDF + PP), vortex mesh of about 33 M DOFs; set 0 stays unless another is faster by more
// than 1 %).
//   p=1 MHD_PP_CFG (256, 4); MHD_SIG_CFG (8, 8, 3): 1.5187 ms  <- chosen
//   p=1 MHD_PP_CFG (256, 4); MHD_SIG_CFG (8, 8, 4): 1.5093 ms
//   p=1 MHD_PP_CFG (256, 4); MHD_SIG_CFG (8, 4, 4): 1.5383 ms
//   p=1 MHD_PP_CFG (128, 8); MHD_SIG_CFG (8, 8, 3): 1.5113 ms
#ifndef MHD_PP_CFG1
#define MHD_PP_CFG1 256, 4
#endif
#ifndef MHD_SIG_CFG1
#define MHD_SIG_CFG1 8, 8, 3
#endif
//   p=2 MHD_PP_CFG (256, 4); MHD_SIG_CFG (8, 4, 3): 1.6700 ms  <- chosen
//   p=2 MHD_PP_CFG (256, 4); MHD_SIG_CFG (8, 4, 4): 1.6682 ms
//   p=2 MHD_PP_CFG (256, 4); MHD_SIG_CFG (4, 4, 4): 1.6936 ms
//   p=2 MHD_PP_CFG (128, 8); MHD_SIG_CFG (8, 4, 3): 1.7097 ms
#ifndef MHD_PP_CFG2
#define MHD_PP_CFG2 256, 4
#endif
#ifndef MHD_SIG_CFG2
#define MHD_SIG_CFG2 8, 4, 3
#endif
//   p=3 MHD_PP_CFG (256, 4); MHD_SIG_CFG (4, 4, 2): 2.6317 ms
//   p=3 MHD_PP_CFG (256, 4); MHD_SIG_CFG (4, 4, 4): 2.5707 ms  <- chosen
//   p=3 MHD_PP_CFG (256, 4); MHD_SIG_CFG (4, 4, 3): 2.5868 ms
//   p=3 MHD_PP_CFG (128, 8); MHD_SIG_CFG (4, 4, 2): 2.6382 ms
#ifndef MHD_PP_CFG3
#define MHD_PP_CFG3 256, 4
#endif
#ifndef MHD_SIG_CFG3
#define MHD_SIG_CFG3 4, 4, 4
#endif
