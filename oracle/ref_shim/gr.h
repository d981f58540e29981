// TEST INFRASTRUCTURE ONLY -- physcon.cpp includes "gr.h", which the reference tree
// does not ship; everything that file needs is declared by physcon.h beside it.
#pragma once
