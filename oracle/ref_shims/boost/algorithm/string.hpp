// Test-infrastructure shim (oracle build only): the reference includes this
// header but calls nothing from it.
#pragma once
