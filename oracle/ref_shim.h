/*
 * Force-included (-include) when compiling the reference's own sources with
 * g++ on Linux.  The reference was written against MSVC/Xcode: it relies on
 * <cmath>/<cfloat>/<cstring> arriving transitively, on MSVC's _ASSERT/_ASSERTE
 * macros (Types.h:38-42 maps DC_BREAK_IF to them) and on a forward
 * declaration of RectanglePacker that MSVC tolerates.  Test infrastructure
 * only.
 */
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>
using std::isnan;
static inline void relight_shim_assert(bool) {}
#define _ASSERTE(x) relight_shim_assert(!!(x))
#define _ASSERT(x) relight_shim_assert(!!(x))
namespace relight { template <typename T> class RectanglePacker; }
