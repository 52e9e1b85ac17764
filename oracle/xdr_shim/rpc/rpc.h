/* the part of <rpc/rpc.h> the reference's writer uses: the XDR shim */
#include "xdr.h"
