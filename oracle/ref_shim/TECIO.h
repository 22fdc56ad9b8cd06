/* No-op stand-in for the Tecplot TecIO header included by the reference's
 * include/mac2d.h.  Result files are out of scope; every call returns 0.
 * Test infrastructure only. */
#ifndef ASD2_REF_SHIM_TECIO_H
#define ASD2_REF_SHIM_TECIO_H
typedef int INTEGER4;
template <class... A> inline INTEGER4 TECINI142(A...) { return 0; }
template <class... A> inline INTEGER4 TECZNE142(A...) { return 0; }
template <class... A> inline INTEGER4 TECDAT142(A...) { return 0; }
template <class... A> inline INTEGER4 TECFIL142(A...) { return 0; }
template <class... A> inline INTEGER4 TECEND142(A...) { return 0; }
#endif
