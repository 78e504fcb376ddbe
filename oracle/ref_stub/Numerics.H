// Empty on purpose: the oracle's reference build defines `Numerics` as a type
// alias in the enclosing namespace before it includes Source/make_rhs.H,
// whose `#include "Numerics.H"` then resolves here.
#pragma once
