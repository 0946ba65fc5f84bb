/* Oracle build stub: stands in for the absent MKL umbrella header.
 * The reference's hot-path sources only need the MKL_INT typedef and,
 * through this header, the x86 pause intrinsic used by its spin loops.
 * No MKL routine is declared; nothing linked against this stub can call MKL. */
#pragma once
#include <immintrin.h>
#include "mkl_types.h"
