/* Oracle build stub for the reference's CMake-generated config.h: every
 * optional USE_* feature is left undefined. */
#pragma once
