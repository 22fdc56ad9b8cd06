/* empty: see TECIO.h */
#include "TECIO.h"
