// Host post-processing of the transient results: the two modules the reference's
// pipeline runs after CalcNonstat3DLine in 3D-only direct mode.
#pragma once
#include <string>

namespace tdem {

// SumNonstat3DOnly (SumNonstat3DOnly/main.cpp:171-384): the per-transmitter result
// files ball_anom.N, edsall_anom.N and eall_anom.N are split into one file per
// component (Bxall.N, Byall.N, Bzall.N, Edsxall.N, Edsyall.N, Edsall.N, Exall.N,
// Eyall.N, Ezall.N) with columns t (ms), normal part (0), anomalous part, total.
// Returns "" or the error (missing or truncated input, unwritable output).
std::string split_components(const std::string& dir);

// SummatorEDMN (SummatorEDMN/main.cpp:37-294): the voltage of every receiver line
// MN of one transmitter, dV(t) = sum over the line's points of E(t) . dl, from
// exall<profile>_<place> / eyall.. / ezall.., the line ends xyzmn<place+1>_<profile>
// and the points xyzVectorElin<place+1>_<profile>; written to edmnall<profile>_<place>
// and, with with_ddv, the difference of the line's halves to edmoonall<profile>_<place>.
// Nothing is done when the file xyzmn lists no lines.
std::string line_voltages(const std::string& dir, bool with_ddv, int profile, int place);

}  // namespace tdem
