// Minimal stand-in for Assimp post-process flags (see scene.h in this folder).
#pragma once
enum aiPostProcessSteps { aiProcess_Triangulate = 0x8, aiProcess_FindDegenerates = 0x10000 };
