// Empty stand-in: the reference includes this header but the PMG path uses nothing from it.
#pragma once
