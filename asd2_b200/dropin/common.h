// Enumerations of the reference's include/common.h:4-11, same names, order
// and values (they are part of the solver interfaces).
#ifndef __COMMON_H_
#define __COMMON_H_

enum class TIMEORDERENUM { EULER, RK2, RK3 };
enum class BC2D { PERIODIC, NEUMANN, DIRICHLET, AXISYM, WALL, INLET, OUTLET, PRESSURE, LSFREE, CUSTOM };
enum class BC3D { PERIODIC, NEUMANN, DIRICHLET, WALL, INLET, OUTLET, PRESSURE, LSFREE, CUSTOM };
enum class PLTTYPE { ASCII, BINARY, BOTH, NONE };
enum class POISSONTYPE { MKL, CG, GS, BICGSTAB, ICPCG };
enum class GAXISENUM2D { X, Y, Z };
enum class GAXISENUM2DAXISYM { R, Z };
enum class GAXISENUM3D { X, Y, Z };

#endif
