// Project-written stand-in for stb_image_write (oracle build only). The
// reference writes 8-bit RGBA PNGs from rainbow-core/file_system.cpp:17-24; this
// replacement writes the RGB channels as a binary PPM to the same file name.
#pragma once

#include <cstdio>

int stbi_write_png(const char* name, int w, int h, int comp, const void* data, int stride);

#ifdef STB_IMAGE_WRITE_IMPLEMENTATION
int stbi_write_png(const char* name, int w, int h, int comp, const void* data, int /*stride*/)
{
	FILE* f = std::fopen(name, "wb");
	if (f == nullptr) return 0;
	std::fprintf(f, "P6\n%d %d\n255\n", w, h);
	const unsigned char* p = static_cast<const unsigned char*>(data);
	for (int i = 0; i < w * h; i++) std::fwrite(p + static_cast<long>(i) * comp, 1, 3, f);
	std::fclose(f);
	return 1;
}
#endif
