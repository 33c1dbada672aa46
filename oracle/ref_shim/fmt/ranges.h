// Shim: local_pointer_chasing.cpp includes fmt only for logging, which the
// single-rank oracle build does not use.
#pragma once
