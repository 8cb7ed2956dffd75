// gls_mtl_image.hpp — TEST INFRASTRUCTURE ONLY. SURF.hpp names Metal
// textures in declarations only; the pin harness runs no Metal host code.
#pragma once

#include <memory>

#include "gls_image.hpp"

namespace gls {
template <class T>
struct mtl_image_2d {
    typedef std::unique_ptr<mtl_image_2d<T>> unique_ptr;
};
}  // namespace gls
