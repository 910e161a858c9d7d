// Empty stand-in: the reference includes <boost/chrono/include.hpp> (include/frechet.hpp:3,
// src/frechet.cpp:7) but uses only std::chrono; boost is not installed here.
#pragma once
