// The reference's poisson2d.h pulls in Intel MKL for its CSR solver types.
// The B200 drop-in needs only the index type used in those signatures.
#ifndef ASD2_DROPIN_MKL_TYPES_H
#define ASD2_DROPIN_MKL_TYPES_H
#ifndef MKL_INT
typedef int MKL_INT;
#endif
#endif
