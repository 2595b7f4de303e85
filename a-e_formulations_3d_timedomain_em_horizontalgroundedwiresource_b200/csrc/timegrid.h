// Host preparation of the time grid: the two modules the reference's pipeline
// runs before the transient solve (GeoCalculatorSP.cpp:2111-2126).
#pragma once
#include <string>

namespace tdem {

// TimeDirectSolver (TimeDirectSolver/main.cpp, TimeStep.cpp:31-130): the times of
// infite.0 become a piecewise-uniform grid whose step grows by the factor in file
// tcff from one interval to the next; infite.0 is rewritten (the old one kept as
// !infite.0) and the source functions currentfunction and deltafunction are
// interpolated onto the new times (old ones kept as !currentfunction, !deltafunction).
std::string time_direct_solver(const std::string& dir);

// CorrectTimeMesh (CorrectTimeMesh/main.cpp): decades (runs of equal steps) that
// are too short for their step are replaced by steps of the previous decade's size;
// infite.0, deltafunction and currentfunction are rewritten on the corrected times
// (old ones kept as !!infite.0, !!deltafunction, !!currentfunction), both function
// files carrying deltafunction's values.
std::string correct_time_mesh(const std::string& dir);

}  // namespace tdem
