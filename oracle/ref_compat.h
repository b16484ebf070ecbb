/* Force-included compatibility header for compiling the PSST reference sources
 * with g++ exactly where they lie (nothing is copied or edited).
 *
 * TEST INFRASTRUCTURE ONLY: this file belongs to the oracle (the checker). The
 * product library never includes or links anything under oracle/.
 *
 * The reference was written for MSVC:
 *  - it throws `std::exception("message")`, a constructor only MSVC provides
 *    (e.g. psstFiniteVolumeGrid.cpp:42, psstConvectiveFlow.cpp:285);
 *  - some translation units rely on headers that MSVC pulls in transitively
 *    (<string> in psstFiniteVolumeGridTools.h:345, <cmath> in
 *    psstGradCalculation.cpp:65).
 * The CP1251 identifier in psstFiniteVolumeGridTools.h:155 is handled by the
 * compiler flag -finput-charset=cp1251, not here.
 *
 * All standard headers the reference uses are included first, then the name
 * `exception` is redirected to a runtime_error subclass that accepts a message.
 * Headers included after this point are already guarded, so the macro only
 * affects the reference's own code.
 */
#ifndef PSST_REF_COMPAT_H
#define PSST_REF_COMPAT_H
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <vector>

namespace std {
struct psst_msvc_exception : public runtime_error {
    psst_msvc_exception() : runtime_error("exception") {}
    explicit psst_msvc_exception(const char *msg) : runtime_error(msg) {}
};
}  // namespace std

#define exception psst_msvc_exception
#endif
