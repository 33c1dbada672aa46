// Shim: logging is not used by the compiled oracle path.
#pragma once
