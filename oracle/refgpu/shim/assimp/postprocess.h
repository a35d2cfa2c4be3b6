// Stand-in: mesh import is off the grid step; the reference only names
// these types in declarations.
#pragma once
struct aiNode;
struct aiScene;
