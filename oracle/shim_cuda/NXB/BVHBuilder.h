// ORACLE / TEST INFRASTRUCTURE ONLY: see BVH.h in this directory.
#pragma once
#include "BVH.h"
