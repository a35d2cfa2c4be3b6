// Empty stand-in: the reference includes it for serialisation, JSON or D3D11
// interop, none of which the grid step uses.
#pragma once
