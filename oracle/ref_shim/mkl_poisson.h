/* empty: everything the reference uses is declared in mkl.h */
#include "mkl.h"
