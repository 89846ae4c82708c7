#pragma once
#include "carbon.h"
