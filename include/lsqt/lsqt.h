// Replaces src/lsqt.h: the run over one input directory (src/lsqt.cu:135-152).
#pragma once

#include <string>

#include "lsqt/common.h"

void lsqt(std::string input_directory);
