/* QD 2.3.23 configuration used by the oracle build.
 *
 * This stands in for the header that QD's configure script would generate.
 * It selects the same arithmetic the reference build uses on x86-64
 * (sloppy, Cray-style add; sloppy multiply and divide; no fused
 * multiply-add, so two_prod uses Dekker's split).  Test infrastructure
 * only: the product never links QD.
 */
#ifndef _QD_QD_CONFIG_H
#define _QD_QD_CONFIG_H 1
#define QD_API
#define QD_INLINE 1
#define QD_HAVE_STD 1
#define QD_SLOPPY_MUL 1
#define QD_SLOPPY_DIV 1
/* QD_IEEE_ADD, QD_FMA and QD_FMS are deliberately left undefined. */
#include <cmath>
#define QD_ISNAN(x) std::isnan(x)
#define QD_ISINF(x) std::isinf(x)
#define QD_ISFINITE(x) std::isfinite(x)
#define QD_COPYSIGN(x, y) std::copysign(x, y)
#endif
