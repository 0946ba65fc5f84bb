/* Oracle build stub: the one MKL type the reference's sparse sources use. */
#pragma once
#ifndef MKL_INT
#define MKL_INT int
#endif
