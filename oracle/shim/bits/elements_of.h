// Empty stand-in: only commented-out reference code used std::generator.
#pragma once
