#pragma once
#include "../Preconditioner.h"
