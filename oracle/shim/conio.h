// Empty stand-in for the MSVC console header (oracle build of the reference only).
#pragma once
