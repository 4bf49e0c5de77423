// CHECKER ONLY: see ../cv_stub.hpp
#pragma once
#include "../../cv_stub.hpp"
