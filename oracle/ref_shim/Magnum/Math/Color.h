#pragma once
#include "../Magnum.h"
