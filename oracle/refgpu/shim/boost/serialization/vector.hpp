// Stand-in: only the name boost::serialization::access is referenced.
#pragma once
namespace boost { namespace archive {} namespace serialization { class access {}; } }
