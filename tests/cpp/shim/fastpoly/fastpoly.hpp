// Include redirect: the reference's tests include "fastpoly/fastpoly.hpp"; with this
// directory first on the include path they compile unchanged against the B200
// drop-in header (oracle/Makefile, target ref-tests).
#include "fpx/fastpoly.hpp"
