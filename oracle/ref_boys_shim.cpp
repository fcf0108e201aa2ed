// C entry point around the reference's own Boys function
// (src/lookup/boys.cpp:1592-1618), compiled from the reference sources in
// place by oracle/build_ref.sh.  Test infrastructure only: it produces the
// golden Boys values in tests/golden/boys_ref.json.
#include "lookup/boys.h"

extern "C" double ref_boys(int n, double x)
{
    return HartreeFock::Lookup::boys(n, x);
}
