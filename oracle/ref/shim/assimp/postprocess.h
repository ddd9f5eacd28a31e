#pragma once
enum { aiProcess_Triangulate = 0x8 };
