#pragma once
#include "Windows.h"
