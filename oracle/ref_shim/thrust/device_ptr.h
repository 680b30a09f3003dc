// thrust stand-in header: everything the reference uses is in thrust/copy.h.
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include "copy.h"
