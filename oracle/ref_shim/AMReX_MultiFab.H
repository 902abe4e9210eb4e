#include "AMReX.H"
