/* qop_config.h for the reference build against qdp_shim: the configure
   options of a plain single-process CPU build (no QLL, QUDA, BLAS, LAPACK,
   Nc = N). */
#ifndef QOP_CONFIG_SHIM_H
#define QOP_CONFIG_SHIM_H
#define QOP_VERSION "0.21.1"
#define PACKAGE_VERSION "0.21.1"
#endif
#define VERSION "0.21.1"
