// Empty stand-in for the MSVC file-sharing header (oracle build of the reference only).
#pragma once
