// Empty stand-in for the MSVC low-level I/O header (oracle build of the reference only).
#pragma once
#include <unistd.h>
