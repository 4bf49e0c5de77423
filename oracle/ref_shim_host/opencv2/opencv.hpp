// CHECKER ONLY: see ../cv_host.hpp
#pragma once
#include "../cv_host.hpp"
