// gls_mtl.hpp — TEST INFRASTRUCTURE ONLY. SURF.hpp names the Metal context
// type in declarations only; the pin harness runs no Metal host code.
#pragma once

class MetalContext;
