// Empty on purpose: the oracle's reference build defines `Model` as a type
// alias in the enclosing namespace before it includes Source/make_rhs.H,
// whose `#include "Model.H"` then resolves here.
#pragma once
