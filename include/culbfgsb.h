/*
 * culbfgsb.h -- the reference's C++ surface, reachable without the culbfgsb/ directory
 * prefix: forwards to culbfgsb/culbfgsb.h (the drop-in adapter over lbfgsb_b200.h).
 */
#ifndef LBFGSB_B200_CULBFGSB_FORWARD_H_
#define LBFGSB_B200_CULBFGSB_FORWARD_H_
#include "culbfgsb/culbfgsb.h"
#endif
