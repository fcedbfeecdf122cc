// stb_image implementation unit for the reference builds in oracle/_ref
// (the reference's texture loader calls stbi_loadf / stbi_load).
#define STB_IMAGE_IMPLEMENTATION
#include "stb_image.h"
