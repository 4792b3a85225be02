#include "iga_plan.hpp"
void iga_solver_release(iga_plan *) {}
