/* Empty stand-in: the reference includes <cublas.h> but calls nothing from it. */
#ifndef PFAG_SHIM_CUBLAS_H
#define PFAG_SHIM_CUBLAS_H
#endif
